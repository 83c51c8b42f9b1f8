// Host heap resource (new/delete through the pmr default) for the oracle build.
#pragma once
#include <cstddef>
#include <new>
#include "vecmem/memory/memory_resource.hpp"

namespace vecmem {
class host_memory_resource final : public memory_resource {
   private:
    void* do_allocate(std::size_t bytes, std::size_t align) override {
        return ::operator new(bytes, std::align_val_t(align));
    }
    void do_deallocate(void* p, std::size_t, std::size_t align) override {
        ::operator delete(p, std::align_val_t(align));
    }
    bool do_is_equal(const std::pmr::memory_resource& o) const noexcept override {
        return this == &o;
    }
};
}  // namespace vecmem
