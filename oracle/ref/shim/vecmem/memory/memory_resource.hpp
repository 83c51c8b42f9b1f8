// Host-only stand-in for the vecmem memory-resource interface, written from
// the way detray's headers use it: a polymorphic memory resource handed to
// containers by pointer or reference.  Test infrastructure for the oracle
// build only; never part of the product.
#pragma once
#include <memory_resource>

namespace vecmem {
using memory_resource = std::pmr::memory_resource;
}  // namespace vecmem
