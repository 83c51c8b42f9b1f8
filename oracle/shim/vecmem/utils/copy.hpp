// Host-only copy helper: detray's buffer code names it; the oracle never
// moves data to a device, so nothing here is called.
#pragma once
#include "vecmem/containers/data/vector_buffer.hpp"

namespace vecmem {
class copy {
   public:
    enum class type { host_to_device, device_to_host, host_to_host, unknown };
    template <typename... A>
    copy& setup(A&&...) { return *this; }
    template <typename... A>
    copy& operator()(A&&...) { return *this; }
    struct event_type { void wait() {} };
    using event_ptr = event_type*;
};
}  // namespace vecmem
