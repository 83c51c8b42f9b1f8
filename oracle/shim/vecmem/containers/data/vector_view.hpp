// Non-owning (size, pointer) view, the shape detray's device views expect.
#pragma once
#include <cstddef>
#include <type_traits>

// Device annotations for the CUDA build of the reference's propagator (the
// GPU baseline); empty for the host compilers.
#if defined(__CUDACC__)
#define VECMEM_HOST_AND_DEVICE __host__ __device__
#else
#define VECMEM_HOST_AND_DEVICE
#endif

namespace vecmem::data {
template <typename T>
class vector_view {
   public:
    using size_type = unsigned int;
    using pointer = T*;
    using value_type = T;
    vector_view() = default;
    VECMEM_HOST_AND_DEVICE vector_view(size_type n, pointer p) : m_size(n), m_capacity(n), m_ptr(p) {}
    template <typename U,
              std::enable_if_t<std::is_convertible_v<U*, T*>, bool> = true>
    VECMEM_HOST_AND_DEVICE vector_view(const vector_view<U>& o)
        : m_size(o.size()), m_capacity(o.capacity()), m_ptr(o.ptr()) {}
    VECMEM_HOST_AND_DEVICE size_type size() const { return m_size; }
    VECMEM_HOST_AND_DEVICE size_type capacity() const { return m_capacity; }
    VECMEM_HOST_AND_DEVICE pointer ptr() const { return m_ptr; }
    VECMEM_HOST_AND_DEVICE size_type* size_ptr() const { return nullptr; }

   private:
    size_type m_size{0};
    size_type m_capacity{0};
    pointer m_ptr{nullptr};
};

template <typename T>
class jagged_vector_view {
   public:
    using size_type = unsigned int;
    using value_type = vector_view<T>;
    using pointer = value_type*;
    jagged_vector_view() = default;
    VECMEM_HOST_AND_DEVICE jagged_vector_view(size_type n, pointer p) : m_size(n), m_ptr(p) {}
    template <typename U,
              std::enable_if_t<std::is_convertible_v<U*, T*>, bool> = true>
    VECMEM_HOST_AND_DEVICE jagged_vector_view(const jagged_vector_view<U>& o)
        : m_size(o.size()),
          m_ptr(reinterpret_cast<pointer>(o.ptr())) {}
    VECMEM_HOST_AND_DEVICE size_type size() const { return m_size; }
    VECMEM_HOST_AND_DEVICE size_type capacity() const { return m_size; }
    VECMEM_HOST_AND_DEVICE pointer ptr() const { return m_ptr; }
    VECMEM_HOST_AND_DEVICE pointer host_ptr() const { return m_ptr; }

   private:
    size_type m_size{0};
    pointer m_ptr{nullptr};
};

enum class buffer_type { fixed_size = 0, resizable = 1 };

template <typename T>
class vector_buffer : public vector_view<T> {
   public:
    using vector_view<T>::vector_view;
};

template <typename T>
class jagged_vector_buffer : public jagged_vector_view<T> {};
}  // namespace vecmem::data
