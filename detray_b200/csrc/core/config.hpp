// dprop_config (the C-ABI mirror of propagation::config,
// propagator/propagation_config.hpp:22-40) -> the device-side prop_cfg.
#pragma once

#include "detray_b200/dprop.h"
#include "propagate.cuh"

namespace dprop {

template <typename S>
prop_cfg<S> make_prop_cfg(const dprop_config& c) {
    prop_cfg<S> p{};
    p.step.min_stepsize = static_cast<S>(c.min_stepsize);
    p.step.rk_error_tol = static_cast<S>(c.rk_error_tol);
    p.step.max_rk_updates = c.max_rk_updates;
    p.step.do_covariance_transport = c.do_covariance_transport != 0;
    p.step.field_gradient = c.use_field_gradient != 0;
    p.step.use_mean_loss = c.use_mean_loss != 0;
    p.step.use_eloss_gradient = c.use_eloss_gradient != 0;
    p.step.mass = static_cast<S>(c.mass);
    p.step.electron = (c.pdg == 11 || c.pdg == -11);
    p.nav.isect.min_mask_tol = static_cast<S>(c.min_mask_tolerance);
    p.nav.isect.max_mask_tol = static_cast<S>(c.max_mask_tolerance);
    p.nav.isect.mask_tol_scalor = static_cast<S>(c.mask_tolerance_scalor);
    p.nav.isect.path_tol = static_cast<S>(c.path_tolerance);
    p.nav.isect.overstep_tol = static_cast<S>(c.overstep_tolerance);
    p.nav.isect.min_tol_is_max = (c.min_mask_tolerance == FLT_MAX);
    p.nav.win0 = c.search_window[0];
    p.nav.win1 = c.search_window[1];
    p.act.path_limit = c.use_path_limit_aborter ? static_cast<S>(c.path_limit)
                                                : limits<S>::max();
    p.act.use_path_limit = c.use_path_limit_aborter != 0;
    p.act.use_interactor = c.use_material_interactor != 0;
    p.act.estimate_noise = c.estimate_scattering_noise != 0;
    p.act.n_stddev = static_cast<S>(c.n_scattering_stddev);
    p.act.accumulated_error = static_cast<S>(c.accumulated_error);
    p.act.mass = static_cast<S>(c.mass);
    p.act.electron = (c.pdg == 11 || c.pdg == -11);
    // FLT_MAX in the float config means "unconstrained" in any precision
    p.step_constraint = (c.step_constraint >= FLT_MAX)
                            ? limits<S>::max()
                            : static_cast<S>(c.step_constraint);
    p.record_all = c.record_all_surfaces != 0;
    p.max_records = c.max_records;
    p.max_iterations = c.max_iterations;
    return p;
}

}  // namespace dprop
