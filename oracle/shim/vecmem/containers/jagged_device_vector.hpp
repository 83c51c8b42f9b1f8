#pragma once
#include "vecmem/containers/device_vector.hpp"

namespace vecmem {
template <typename T>
class jagged_device_vector {
   public:
    using size_type = unsigned int;
    jagged_device_vector() = default;
    VECMEM_HOST_AND_DEVICE explicit jagged_device_vector(const data::jagged_vector_view<T>& v)
        : m_view(v) {}
    VECMEM_HOST_AND_DEVICE device_vector<T> operator[](size_type i) const {
        return device_vector<T>(m_view.ptr()[i]);
    }
    VECMEM_HOST_AND_DEVICE device_vector<T> at(size_type i) const { return (*this)[i]; }
    VECMEM_HOST_AND_DEVICE size_type size() const { return m_view.size(); }
    VECMEM_HOST_AND_DEVICE bool empty() const { return m_view.size() == 0; }

   private:
    data::jagged_vector_view<T> m_view;
};
}  // namespace vecmem
