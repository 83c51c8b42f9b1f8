// Host-only stand-in for the vecmem memory-resource interface (vecmem 1.23.0
// is a dependency of detray that is not vendored with it), written from the
// way detray's headers use it: a polymorphic memory resource handed to
// containers by pointer or reference.  Only the host-side tools that compile
// detray headers use these files (the geometry exporter and the oracle
// build); the device library does not.
#pragma once
#include <memory_resource>

namespace vecmem {
using memory_resource = std::pmr::memory_resource;
}  // namespace vecmem
