// Fixed-capacity vector over a view; host-side stand-in for the device vector.
#pragma once
#include <cassert>
#include "vecmem/containers/data/vector_view.hpp"

namespace vecmem {
template <typename T>
class device_vector {
   public:
    using value_type = T;
    using size_type = unsigned int;
    using reference = T&;
    using const_reference = const T&;
    using pointer = T*;
    using const_pointer = const T*;
    using iterator = T*;
    using const_iterator = const T*;
    device_vector() = default;
    VECMEM_HOST_AND_DEVICE explicit device_vector(const data::vector_view<T>& v)
        : m_ptr(v.ptr()), m_size(v.size()), m_capacity(v.capacity()) {}
    VECMEM_HOST_AND_DEVICE reference operator[](size_type i) { return m_ptr[i]; }
    VECMEM_HOST_AND_DEVICE const_reference operator[](size_type i) const { return m_ptr[i]; }
    VECMEM_HOST_AND_DEVICE reference at(size_type i) { return m_ptr[i]; }
    VECMEM_HOST_AND_DEVICE const_reference at(size_type i) const { return m_ptr[i]; }
    VECMEM_HOST_AND_DEVICE size_type size() const { return m_size; }
    VECMEM_HOST_AND_DEVICE size_type capacity() const { return m_capacity; }
    VECMEM_HOST_AND_DEVICE bool empty() const { return m_size == 0; }
    VECMEM_HOST_AND_DEVICE iterator begin() { return m_ptr; }
    VECMEM_HOST_AND_DEVICE iterator end() { return m_ptr + m_size; }
    VECMEM_HOST_AND_DEVICE const_iterator begin() const { return m_ptr; }
    VECMEM_HOST_AND_DEVICE const_iterator end() const { return m_ptr + m_size; }
    VECMEM_HOST_AND_DEVICE pointer data() { return m_ptr; }
    VECMEM_HOST_AND_DEVICE const_pointer data() const { return m_ptr; }
    VECMEM_HOST_AND_DEVICE reference front() { return m_ptr[0]; }
    VECMEM_HOST_AND_DEVICE reference back() { return m_ptr[m_size - 1]; }
    VECMEM_HOST_AND_DEVICE void push_back(const T& v) {
        assert(m_size < m_capacity);
        m_ptr[m_size++] = v;
    }
    VECMEM_HOST_AND_DEVICE size_type push_back_default() { return m_size++; }
    VECMEM_HOST_AND_DEVICE void clear() { m_size = 0; }
    VECMEM_HOST_AND_DEVICE void resize(size_type n) { m_size = n; }

   private:
    pointer m_ptr{nullptr};
    VECMEM_HOST_AND_DEVICE size_type m_size{0};
    VECMEM_HOST_AND_DEVICE size_type m_capacity{0};
};
}  // namespace vecmem
