// vecmem::vector: a std::vector with a polymorphic allocator, plus get_data.
#pragma once
#include <memory_resource>
#include <vector>
#include "vecmem/containers/data/vector_view.hpp"
#include "vecmem/memory/memory_resource.hpp"

namespace vecmem {
template <typename T>
using vector = std::vector<T, std::pmr::polymorphic_allocator<T>>;

template <typename T, typename A>
data::vector_view<T> get_data(std::vector<T, A>& v) {
    return {static_cast<unsigned int>(v.size()), v.data()};
}
template <typename T, typename A>
data::vector_view<const T> get_data(const std::vector<T, A>& v) {
    return {static_cast<unsigned int>(v.size()), v.data()};
}
template <typename T>
data::vector_view<T> get_data(data::vector_buffer<T>& b) {
    return b;
}
template <typename T>
data::vector_view<T> get_data(const data::vector_buffer<T>& b) {
    return b;
}
}  // namespace vecmem
