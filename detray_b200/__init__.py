"""detray-b200: batched charged-track propagation through detray geometries
on one B200 (sm_100a), behind a C ABI that replaces detray's device
propagation call.  See include/detray_b200/dprop.h."""

__all__ = ["abi", "geometry", "propagator", "tracks", "units"]
