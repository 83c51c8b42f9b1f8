/*
 * detray-b200 C ABI: batched charged-track propagation on one B200.
 *
 * This header is the whole drop-in boundary.  It replaces the device side of
 * detray's track propagation, which in the reference is reached through
 *
 *   (i)   detray::get_buffer(det, dev_mr, copy) / detray::get_data(buffer)
 *         core/include/detray/core/detail/container_buffers.hpp:82-195
 *         -> here: dprop_detector_create() from flattened tables;
 *   (ii)  a covfie field view handed to the stepper
 *         tests/include/detray/test/common/bfield.hpp:35-47 (host),
 *         tests/include/detray/test/device/cuda/bfield.hpp:28-32 (device)
 *         -> here: dprop_field_create_const() / dprop_field_create_grid();
 *   (iii) the batch launcher run_propagation_kernel<propagator_t>(cfg,
 *         det_view, field_view, actor_states, tracks, n)
 *         tests/benchmarks/include/detray/benchmarks/device/cuda/
 *         propagation_benchmark.hpp:83-93 and propagation_benchmark.cu:96-118
 *         -> here: dprop_propagate() (device buffers, stream ordered) and
 *            dprop_propagate_host() (host buffers, copies included).
 *
 * The actor chain is the one the reference's device tests compose
 * (tests/include/detray/test/device/propagator_test.hpp:84-93):
 *   pathlimit_aborter -> parameter_updater< pointwise_material_interactor >
 * with the run-time switches of propagation::config
 * (core/include/detray/propagator/propagation_config.hpp:22-40) mirrored in
 * dprop_config.
 *
 * Conventions: plain C types only, no exceptions cross this boundary, every
 * function returns a dprop_status; dprop_last_error() gives the message of
 * the last failure on the calling thread.  Units are detray's: mm, GeV, T
 * expressed in detray's internal unit system (1 T = 0.000299792458 GeV/mm/e).
 */
#ifndef DETRAY_B200_DPROP_H
#define DETRAY_B200_DPROP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPROP_ABI_VERSION 3u

/* ------------------------------------------------------------------ status */
typedef enum dprop_status {
    DPROP_OK = 0,
    DPROP_E_INVALID = 1,   /* bad argument or inconsistent tables          */
    DPROP_E_CUDA = 2,      /* a CUDA runtime call failed                   */
    DPROP_E_NO_DEVICE = 3, /* no usable sm_100 device                      */
    DPROP_E_OOM = 4,       /* device allocation failed                     */
    DPROP_E_TIMEOUT = 5,   /* a bounded device wait ran out                */
    DPROP_E_UNSUPPORTED = 6
} dprop_status;

/* Per-track outcome, written to dprop_results.status.  Mirrors the
 * navigation status reached at the end of propagator::propagate
 * (core/include/detray/propagator/propagator.hpp:389-399) and the abort
 * reasons of the reference (navigation_state.hpp:414-433, aborters.hpp:62-70,
 * propagator.hpp:349-373, navigation_functions.hpp:327-330). */
typedef enum dprop_track_status {
    DPROP_TRK_EXITED = 0,        /* left the world: propagate() returned true */
    DPROP_TRK_PATH_LIMIT = 1,    /* pathlimit_aborter fired                   */
    DPROP_TRK_STALLED = 2,       /* > 10 non-advancing steps                  */
    DPROP_TRK_NO_SURFACE = 3,    /* loose re-initialisation found nothing     */
    DPROP_TRK_MAX_ITER = 4,      /* device iteration budget exhausted         */
    DPROP_TRK_NOT_RUN = 5,       /* never started (e.g. invalid input)        */
    DPROP_TRK_NONFINITE = 6      /* state became NaN/inf                      */
} dprop_track_status;

/* --------------------------------------------------------- detector tables
 * The flattened form of detray::detector<metadata> (core/detector.hpp:57-355).
 * All indices are 0-based positions in the arrays below.  Tables are given
 * in double precision on the host; the library stores its own device copy. */

/* Mask shapes on the path (the headers of geometry/shapes). */
typedef enum dprop_shape {
    DPROP_SHAPE_RECTANGLE = 0,     /* rectangle2D: v0 half_x, v1 half_y                 */
    DPROP_SHAPE_TRAPEZOID = 1,     /* trapezoid2D: v0 hl_x(-y), v1 hl_x(+y), v2 hl_y, v3 1/(2 hl_y) */
    DPROP_SHAPE_RING = 2,          /* ring2D: v0 inner_r, v1 outer_r                    */
    DPROP_SHAPE_CYLINDER = 3,      /* cylinder2D: v0 r, v1 lower_z, v2 upper_z          */
    DPROP_SHAPE_CONCENTRIC_CYL = 4,/* concentric_cylinder2D: v0 r, v1 lower_z, v2 upper_z */
    DPROP_SHAPE_LINE = 5,          /* line (drift cell / straw tube, line.hpp): v0 cell half width or
                                      radius, v1 half_z, v2 square cross-section (1) / circular (0) */
    DPROP_SHAPE_COUNT = 6
} dprop_shape;

/* Surface categories, same values as detray::surface_id
 * (core/include/detray/definitions/geometry.hpp:40-46). */
typedef enum dprop_surface_kind {
    DPROP_SF_PORTAL = 0,
    DPROP_SF_SENSITIVE = 1,
    DPROP_SF_PASSIVE = 2
} dprop_surface_kind;

#define DPROP_INVALID_INDEX 0xffffffffu
#define DPROP_INVALID_LINK 0xffffu

typedef struct dprop_surface_desc {
    uint64_t barcode;       /* geometry::identifier value (identifier.hpp:153-157) */
    uint32_t mask_begin;    /* [mask_begin, mask_end) into masks                   */
    uint32_t mask_end;
    uint32_t transform;     /* into transforms                                     */
    uint32_t material;      /* into slabs (material_kind 0) or into grids, a
                               material map (material_kind 1);
                               DPROP_INVALID_INDEX: no material              */
    uint32_t volume;        /* owning volume                                       */
    uint8_t shape;          /* dprop_shape of all masks of this surface            */
    uint8_t kind;           /* dprop_surface_kind                                  */
    uint8_t material_kind;  /* 0: homogeneous slab / rod, 1: material map          */
    uint8_t pad;
} dprop_surface_desc;

typedef struct dprop_mask_desc {
    double values[6];       /* shape bounds, meaning per dprop_shape               */
    uint32_t volume_link;   /* next volume through this mask, DPROP_INVALID_LINK = leaves world */
    uint32_t pad;
} dprop_mask_desc;

/* Placement: rotation columns (local x, y, z axes in global frame),
 * translation, and the inverse transform as stored by the reference's
 * transform3 (algebra/generic/impl/generic_transform3.hpp). */
typedef struct dprop_transform_desc {
    double rot[9];          /* column-major: x axis, y axis, z axis            */
    double translation[3];
    double inv_rot[9];      /* column-major rotation part of the inverse       */
    double inv_translation[3];
} dprop_transform_desc;

/* Homogeneous material slab (material/material_slab.hpp:78-97) with the
 * derived quantities the interaction formulas read
 * (material/material.hpp, material/detail/relativistic_quantities.hpp). */
typedef struct dprop_slab_desc {
    double thickness;
    double thickness_in_X0;
    double X0;
    double molar_electron_density;  /* Z * molar density                 */
    double mean_excitation_energy;  /* I                                 */
    double density_a, density_m, density_x0, density_x1, density_c;
    uint32_t has_density_effect;
    uint32_t kind;                  /* dprop_material_kind                  */
} dprop_slab_desc;

/* Surface material kinds (material/material_slab.hpp,
 * material/material_rod.hpp). */
typedef enum dprop_material_kind {
    DPROP_MATERIAL_SLAB = 0,  /* thickness t: path t / |cos(incidence)|       */
    DPROP_MATERIAL_ROD = 1    /* rod of radius t around a line surface: path
                                 2 sqrt((t^2 - d^2) / sin^2(incidence)) at
                                 closest approach d, 0 for |d| > t           */
} dprop_material_kind;

typedef enum dprop_grid_kind {
    DPROP_GRID_NONE = 0,
    DPROP_GRID_CYLINDER = 1, /* axes (phi circular [-pi,pi], z closed), ref. radius */
    DPROP_GRID_DISC = 2,     /* axes (r closed, phi circular [-pi,pi])              */
    /* Material maps (material/material_map.hpp: a grid of material slabs over
     * the surface's bound local coordinates, one slab index per bin into
     * slabs, looked up at the track's bound local position by
     * material_accessor::get, material/detail/material_accessor.hpp): */
    DPROP_GRID_MATERIAL_CYLINDER = 3, /* axes (r*phi circular, z closed)         */
    DPROP_GRID_MATERIAL_DISC = 4,     /* axes (r closed, phi circular)           */
    DPROP_GRID_MATERIAL_CARTESIAN = 5 /* axes (x closed, y closed)               */
} dprop_grid_kind;

/* A 2D surface grid of navigation/accelerators/spatial_grid.hpp with
 * regular binning: spatial_grid<..., static_array<surface,1>> (one surface
 * per bin, multi = 0) or spatial_grid<..., dynamic_array<surface>> (several
 * surfaces per bin, multi = 1). */
typedef struct dprop_grid_desc {
    uint32_t kind;          /* dprop_grid_kind                                  */
    uint32_t n_bins[2];
    uint32_t bin_offset;    /* into grid_bins, bins serialised as
                               bin0 + bin1 * n_bins[0].  multi = 0: one entry
                               per bin, a surface index or DPROP_INVALID_INDEX.
                               multi = 1: n_bins[0]*n_bins[1] + 1 entries;
                               entries b and b+1 are the [begin, end) positions
                               in grid_bins of bin b's surface indices          */
    uint32_t transform;     /* grid placement (the volume's transform)          */
    uint32_t multi;
    double axis_min[2];
    double axis_max[2];
    double radius;          /* reference cylinder radius (DPROP_GRID_CYLINDER)  */
} dprop_grid_desc;

typedef struct dprop_volume_desc {
    uint32_t transform;
    uint32_t bf_begin;      /* [bf_begin, bf_end) into bf_surfaces: portals and
                               passives searched by brute force                 */
    uint32_t bf_end;
    uint32_t grid;          /* into grids, or DPROP_INVALID_INDEX                */
    uint32_t material;      /* homogeneous volume material: into slabs (kind
                               DPROP_MATERIAL_SLAB; thickness unused), the
                               material the stepper's energy loss dq/p/ds
                               reads (tracking_volume::material_parameters,
                               rk_stepper.hpp:148-231); DPROP_INVALID_INDEX:
                               none                                         */
} dprop_volume_desc;

typedef struct dprop_detector_desc {
    uint32_t abi_version;           /* = DPROP_ABI_VERSION */
    uint32_t n_volumes, n_surfaces, n_masks, n_transforms, n_slabs;
    uint32_t n_bf_surfaces, n_grids, n_grid_bins;
    const dprop_volume_desc* volumes;
    const dprop_surface_desc* surfaces;
    const dprop_mask_desc* masks;
    const dprop_transform_desc* transforms;
    const dprop_slab_desc* slabs;
    const uint32_t* bf_surfaces;    /* surface indices                          */
    const dprop_grid_desc* grids;
    const uint32_t* grid_bins;      /* surface index or DPROP_INVALID_INDEX      */
} dprop_detector_desc;

typedef struct dprop_detector dprop_detector;
typedef struct dprop_field dprop_field;

/* ------------------------------------------------------------------ config
 * Mirrors propagation::config = {navigation, stepping} and the actor chain
 * switches.  Defaults (dprop_config_default) are the reference's defaults:
 * stepping_config.hpp:27-77, navigation_config.hpp:23-56,
 * intersection_config.hpp:20-33. */
typedef struct dprop_config {
    /* stepping::config */
    float min_stepsize;
    float rk_error_tol;
    float step_constraint;
    float path_limit;
    uint32_t max_rk_updates;
    uint8_t use_mean_loss;
    uint8_t use_eloss_gradient;
    uint8_t use_field_gradient;  /* transport Jacobian with the field's
                                    gradient (d(pos)/d(pos0), d(dir)/d(pos0)
                                    from central differences of the field,
                                    rk_stepper.hpp:872-997): plain method and
                                    adjoint mode, 64 registers; the
                                    persistent method and the direct
                                    navigator reject it                   */
    uint8_t do_covariance_transport;
    /* intersection::config */
    float min_mask_tolerance;
    float max_mask_tolerance;
    float mask_tolerance_scalor;
    float path_tolerance;
    float overstep_tolerance;
    /* navigation::config */
    uint32_t search_window[2];
    float accumulated_error;
    int32_t n_scattering_stddev;
    uint8_t estimate_scattering_noise;
    /* actor chain */
    uint8_t use_path_limit_aborter;   /* pathlimit_aborter in the chain        */
    uint8_t use_material_interactor;  /* pointwise_material_interactor        */
    uint8_t record_all_surfaces;      /* 0: record surfaces the transporter
                                         visits (sensitive or with material);
                                         1: also portals/passives w/o material */
    /* particle hypothesis (muon by default, charge sign follows q/p) */
    float mass;
    int32_t pdg;
    /* device limits */
    uint32_t max_records;             /* per-track record capacity            */
    uint32_t max_iterations;          /* A/N/S loop bound per track           */
} dprop_config;

/* ------------------------------------------------------------------ tracks
 * Struct-of-arrays free track parameters, detray's free vector layout
 * [x, y, z, t, tx, ty, tz, q/p] (definitions/track_parametrization.hpp:49-63).
 * Device-side float arrays for dprop_propagate; host double arrays for
 * dprop_propagate_host. */
typedef struct dprop_tracks {
    const void* pos[3];
    const void* time;
    const void* dir[3];
    const void* qop;
} dprop_tracks;

/* Results.  Records are laid out slot-major: record k of track t sits at
 * index k * n_tracks + t, so that lanes of a warp writing the same slot
 * coalesce.  Bound parameters follow detray's bound vector
 * [loc0, loc1, phi, theta, q/p, t]; the covariance is the upper triangle of
 * the 6x6 matrix, row by row (21 values). */
typedef struct dprop_results {
    uint8_t* status;          /* [n] dprop_track_status                        */
    uint32_t* n_records;      /* [n] records written (may exceed capacity: then
                                  only the first max_records are stored)        */
    uint32_t* n_steps;        /* [n] accepted RK steps                          */
    uint32_t* n_trials;       /* [n] RK trials                                  */
    void* path_length;        /* [n] final path length                          */
    void* final_free[8];      /* [n] each; may be NULL                          */
    uint64_t* rec_barcode;    /* [max_records * n]                              */
    void* rec_bound[6];       /* [max_records * n] each; may be NULL            */
    void* rec_cov[21];        /* [max_records * n] each; may be NULL            */
    void* rec_path;           /* [max_records * n]; may be NULL                 */
    uint8_t* rec_flags;       /* [max_records * n]; bit0: transported (bound +
                                  cov valid), bit1: portal, bit2: material     */
    uint32_t* n_intersections;/* [n] ray-surface intersections evaluated;
                                  may be NULL                                  */
    uint32_t* n_transports;   /* [n] covariance transports to a surface;
                                  may be NULL                                  */
    uint32_t* n_material;     /* [n] material interactions; may be NULL        */
    uint64_t* rec_offsets;    /* host entry point only: if not NULL, records
                                  are returned as a jagged array - the records
                                  of track t are entries [rec_offsets[t],
                                  rec_offsets[t+1]) of the rec_* arrays (at
                                  most max_records per track, n + 1 offsets),
                                  and only stored records are copied back     */
} dprop_results;

/* Launch shape; zero fields pick the library defaults / autotuned values. */
typedef enum dprop_method {
    DPROP_METHOD_PLAIN = 0,      /* one thread per track, whole propagation   */
    DPROP_METHOD_PERSISTENT = 1  /* round-based phase kernels: each track's
                                    state lives in device memory between
                                    rounds; every round a queue builder
                                    sorts the live tracks into the work
                                    queues of the step phase (RK steps,
                                    high-trust navigation, path-limit
                                    aborter, surface actors) and the
                                    navigation phase (cache re-evaluation,
                                    volume switch), in direction order, and
                                    persistent
                                    grid-stride kernels pull their tracks
                                    from those queues; after `rounds` rounds
                                    the tracks still alive finish in one
                                    kernel.  Identical results to the plain
                                    form                                      */
} dprop_method;

typedef struct dprop_launch {
    uint32_t method;             /* dprop_method                               */
    uint32_t block_size;         /* threads per CTA.  Plain method: a multiple
                                    of 32 up to 256, 0 = 128 (the register
                                    budget stays the one ctas_per_sm names).
                                    Persistent method: 0 or 128                */
    uint32_t ctas_per_sm;        /* register budget: resident CTAs of 128
                                    threads per SM the kernel is compiled for.
                                    Plain method: 8 (64 registers), 12 (40)
                                    or 16 (32); 0 = 12.  Persistent method,
                                    its step phase: 3 (168 registers), 4
                                    (128) or 5 (102); 0 = 4.  fp64 plain: 8
                                    or 12 (0 = 8); fp64 persistent: 2 (255
                                    registers) or 3 (168); 0 = 2              */
    uint32_t sort_tracks;        /* 1: process tracks ordered by direction
                                    (theta, phi) so that the lanes of a warp
                                    follow similar paths; results are still
                                    written at each track's input position    */
    uint32_t use_graph;          /* 1: capture the whole propagate call into a
                                    CUDA graph on first use and replay it on
                                    later calls with identical arguments       */
    uint32_t precision;          /* 0 or 4: fp32 arithmetic, float track
                                    arrays and results (the default);
                                    8: fp64 end to end - double track arrays,
                                    double arithmetic and double results (the
                                    reference's full-fp64 build); the plain
                                    or the persistent method, use_graph
                                    ignored.  Device API (dprop_propagate)
                                    only                                       */
    /* Persistent method only (0: the library default of each): */
    uint32_t steps_per_round;    /* RK steps a track takes per round at most
                                    (default 16)                               */
    uint32_t rounds;             /* rounds of the phase kernels before the
                                    tracks still alive finish in one kernel
                                    (default 64)                               */
    uint32_t yield_lanes;        /* tracks per warp: a warp of the step phase
                                    ends its round once fewer than this many of
                                    its 32 lanes can still step (default 16)   */
    uint32_t sort_interval;      /* re-sort the live tracks of both phases by
                                    volume every sort_interval rounds (0:
                                    never, the default)                       */
    uint32_t tail_tracks;        /* once fewer tracks than this are alive at
                                    the start of a round, that round runs
                                    them to their end (0: n_tracks / 64;
                                    1: only after `rounds` rounds)            */
    uint32_t reserved[1];
} dprop_launch;

/* ------------------------------------------------------------------ API */
uint32_t dprop_abi_version(void);
const char* dprop_last_error(void);

void dprop_config_default(dprop_config* cfg);

/* Replaces detray::get_buffer + get_data for the detector stores. */
dprop_status dprop_detector_create(const dprop_detector_desc* desc,
                                   int device, dprop_detector** out);
dprop_status dprop_detector_destroy(dprop_detector* det);

/* Constant field, like covfie::backend::constant (bfield.hpp:35-40). */
dprop_status dprop_field_create_const(double bx, double by, double bz,
                                      int device, dprop_field** out);
/* Field map on a regular (r, phi, z) grid, values (Br, Bphi, Bz) per node,
 * node index ((iz * n_phi) + iphi) * n_r + ir; trilinear interpolation with
 * clamping at the grid edges.  Stands where the reference plugs a covfie
 * affine<linear<clamp<strided<...>>>> view (bfield.hpp:43-47). */
dprop_status dprop_field_create_grid(const double* r_phi_z_min,
                                     const double* r_phi_z_max,
                                     const uint32_t* n_r_phi_z,
                                     const float* values, int device,
                                     dprop_field** out);
dprop_status dprop_field_destroy(dprop_field* field);

/* Propagate n tracks whose parameters and results live in device memory.
 * Stream ordered; returns once the work is enqueued on `stream`
 * (a cudaStream_t, or NULL for the legacy default stream). */
dprop_status dprop_propagate(const dprop_config* cfg,
                             const dprop_launch* launch,
                             const dprop_detector* det,
                             const dprop_field* field,
                             const dprop_tracks* tracks,
                             const dprop_results* results, uint64_t n_tracks,
                             void* stream);

/* Same, with host inputs (double precision, as dprop_tracks) and host
 * outputs (the result pointers then point to host memory, with the same
 * element types as on the device).  Copies in, propagates, copies out and
 * synchronises.  Uses library-owned device scratch, grown on demand.  With
 * jagged records (rec_offsets) the batch runs in chunks of up to 256 Ki
 * tracks on four streams, each chunk with the launch's method, sort and
 * register budget (use_graph is ignored there). */
dprop_status dprop_propagate_host(const dprop_config* cfg,
                                  const dprop_launch* launch,
                                  const dprop_detector* det,
                                  const dprop_field* field,
                                  const dprop_tracks* tracks,
                                  const dprop_results* results,
                                  uint64_t n_tracks);

/* ------------------------------------------------------ direct navigation
 * Propagation along a given sequence of surfaces (the Kalman-filter fit and
 * smoothing steps either side of the propagation path): replaces the
 * reference's propagator<rk_stepper, direct_navigator, actor chain>
 * (core/include/detray/navigation/direct_navigator.hpp:34-304) fed by the
 * surface_sequencer actor (core/include/detray/propagator/actors/
 * surface_sequencer.hpp:24-106).
 *
 * The sequence of a track is what the sequencer collects: the sensitive and
 * material surfaces the caching navigator reached, i.e. the records of a
 * dprop_propagate run with record_all_surfaces = 0 - rec_barcode and
 * n_records of that run can be passed as they are.  The navigator
 * intersects only the next surface of the sequence, with every mask
 * accepting the track, and the actor chain (transport, material
 * interaction, records) runs on each of them.  direction -1 walks the
 * sequence from its last entry to its first with the track moving backwards
 * (energy gained in material).  A track whose next surface cannot be
 * intersected ends with DPROP_TRK_NO_SURFACE; an empty sequence ends at
 * once with DPROP_TRK_EXITED and no records. */
typedef struct dprop_sequence {
    const uint64_t* barcodes;   /* [max_length * n]: entry k of track t at
                                   k * n + t (device memory)                   */
    const uint32_t* length;     /* [n] entries per track; values above
                                   max_length are read as max_length          */
    uint32_t max_length;
    int32_t direction;          /* +1 forward, -1 backward                    */
    /* Optional start on a surface (bound_track_parameters: the propagator
     * state converts them to the free vector there, base_stepper.hpp:84-107)
     * instead of dprop_tracks: NULL start_barcode = start from the tracks. */
    const uint64_t* start_barcode;  /* [n] surface of the bound start         */
    const float* start_bound[6];    /* [n] each: loc0, loc1, phi, theta, q/p,
                                       t                                      */
} dprop_sequence;

/* Device buffers, float tracks and results as dprop_propagate; `tracks` may
 * be NULL when the sequence carries a bound start.  Stream ordered. */
dprop_status dprop_propagate_direct(const dprop_config* cfg,
                                    const dprop_detector* det,
                                    const dprop_field* field,
                                    const dprop_tracks* tracks,
                                    const dprop_sequence* sequence,
                                    const dprop_results* results,
                                    uint64_t n_tracks, void* stream);

/* ------------------------------------------------------------ helix scan
 * Truth intersections for navigation validation: each track's exact helix
 * in the constant field b, intersected with every surface of the detector
 * (Newton-Raphson with bisection safeguard), the intersections inside a mask
 * and along the track sorted by path length and cut after the first one that
 * leaves the world.  Replaces the reference's CPU detector scan
 * detector_scanner::run<helix_scan> (tests/include/detray/test/validation/
 * detector_scanner.hpp:52-140) with its helix intersectors
 * (core/include/detray/navigation/intersection/helix_*_intersector.hpp,
 * core/include/detray/utils/root_finding.hpp); the reference's extra start
 * record (a marker at the track origin) is not written.
 *
 * Mask tolerance: mask_tolerance mm on sensitive and passive surfaces, none
 * on portals, as the reference scanner.  The scan is brute force: its cost
 * is n_tracks x n_surfaces root searches. */
typedef enum dprop_scan_status {
    DPROP_SCAN_OK = 0,
    DPROP_SCAN_OVERFLOW = 1,  /* more intersections than capacity: n_hits
                                 holds the number found, nothing is stored  */
    DPROP_SCAN_EMPTY = 2      /* no intersection at all                     */
} dprop_scan_status;

typedef struct dprop_scan_results {
    uint8_t* status;          /* [n] dprop_scan_status                         */
    uint32_t* n_hits;         /* [n] intersections stored                      */
    uint64_t* barcode;        /* [capacity * n]: hit k of track t at k * n + t */
    void* path;               /* [capacity * n] path length along the helix    */
    void* loc[2];             /* [capacity * n] each: bound local coordinates
                                 of the hit; may be NULL                       */
    uint16_t* volume_link;    /* [capacity * n]: volume behind the hit mask,
                                 DPROP_INVALID_LINK leaves the world           */
    uint32_t capacity;
    uint32_t precision;       /* 4: float tracks and results, 8: double        */
} dprop_scan_results;

/* Device buffers (tracks in the precision of `results`), stream ordered. */
dprop_status dprop_helix_scan(const dprop_detector* det, const double b[3],
                              const dprop_tracks* tracks, uint64_t n_tracks,
                              double mask_tolerance,
                              const dprop_scan_results* results,
                              void* stream);

/* Navigation validation against the scan (the comparison of
 * tests/include/detray/test/validation/navigation_validation_utils.hpp:
 * 379-800, per track): `records` are the results of a propagation of the
 * same tracks with record_all_surfaces = 1 (status, n_records, rec_barcode
 * and rec_path used; rec_path in float for record_precision 4, double for
 * 8; max_records its capacity).  A truth surface is missed if no record of
 * it (for portals: of any portal - two portals coincide at a volume
 * boundary and the navigator records one) lies within path_tolerance mm of
 * its path; the truth's final world-exit portal counts as reached when the
 * track exited.  A record is extra if no truth surface matches it. */
typedef struct dprop_validation {
    uint32_t* n_missed;   /* [n] truth surfaces the navigation missed        */
    uint32_t* n_extra;    /* [n] recorded surfaces not on the helix          */
} dprop_validation;

dprop_status dprop_validate_navigation(const dprop_scan_results* truth,
                                       const dprop_results* records,
                                       uint32_t record_precision,
                                       uint32_t max_records,
                                       uint64_t n_tracks,
                                       double path_tolerance,
                                       const dprop_validation* out,
                                       void* stream);

/* ------------------------------------------------- allocation-free variant
 * dprop_propagate_noalloc has no counterpart in the reference.
 *
 * It is for callers that must not have the library allocate device memory
 * while they run: an event-processing framework that hands all device memory
 * to its own pool allocator, a trigger or other latency-bound loop in which a
 * cudaMalloc or cudaFree (which can synchronise the whole device) is not
 * acceptable, or an application that fixes its device-memory budget up
 * front.  It does what dprop_propagate does with sort_tracks = 1 and the
 * plain one-thread-per-track kernel, but the scratch the direction sort needs
 * (keys, indices, radix-sort temporary storage) lives in one fixed array
 * compiled into the library: DPROP_NOALLOC_SCRATCH_BYTES on every GPU that
 * loads the library, held until the process exits.  Inputs and outputs are
 * device buffers passed by the caller, as for dprop_propagate.
 *
 *  - At most DPROP_NOALLOC_MAX_TRACKS tracks per call; a larger batch is
 *    rejected with DPROP_E_INVALID (split it into several calls).
 *  - Each call outside a stream capture looks up the device's copy of the
 *    array (a call inside a capture reuses the last address found on that
 *    device); make the first call on a device before capturing any stream
 *    into a CUDA graph, and call again outside a capture after a
 *    cudaDeviceReset.
 *  - Every call uses the same array: calls whose GPU work overlaps (for
 *    instance on two streams at once) race on it, so the caller must order
 *    them, e.g. by issuing them on one stream.
 */
#define DPROP_NOALLOC_MAX_TRACKS 262144u
#define DPROP_NOALLOC_SCRATCH_BYTES (6u * 1024u * 1024u)
dprop_status dprop_propagate_noalloc(const dprop_config* cfg,
                                     const dprop_detector* det,
                                     const dprop_field* field,
                                     const dprop_tracks* tracks,
                                     const dprop_results* results,
                                     uint64_t n_tracks, void* stream);

/* Autotuner: times candidate launch forms - the plain kernel at the three
 * register budgets (ctas_per_sm 8, 12, 16) with the direction sort, at 16
 * with 256-thread blocks and at 16 without the sort; the persistent method
 * with and without the sort over its step-phase register budget
 * (ctas_per_sm 3, 4, 5), steps per round, tracks per warp (yield_lanes 8,
 * 12, 16), the volume re-sort interval (0, 1, 2) and the number of rounds
 * before the tail kernel - on the first min(n_tracks, 1048576) of the given
 * device tracks (under a CUDA graph if launch->use_graph is set), and writes
 * the fastest into *launch (method, block_size, ctas_per_sm, sort_tracks,
 * steps_per_round, yield_lanes, rounds, sort_interval; use_graph is left as
 * given).  If timings_ms is not NULL it receives one time per candidate
 * (DPROP_AUTOTUNE_CANDIDATES entries).  Allocates temporary device result
 * buffers for the trial runs. */
#define DPROP_AUTOTUNE_CANDIDATES 13
dprop_status dprop_autotune(const dprop_config* cfg, const dprop_detector* det,
                            const dprop_field* field,
                            const dprop_tracks* tracks, uint64_t n_tracks,
                            dprop_launch* launch, float* timings_ms,
                            void* stream);

/* Frees the device memory the library keeps between calls: the cached CUDA
 * graphs (use_graph) with the scratch each owns, and the grow-only scratch
 * of the direction sort, the persistent method and the host-buffer entry
 * points.  Synchronises the current device first; no propagate call may be
 * running on another host thread.  Later calls allocate again on demand.
 * Counterpart of releasing the vecmem buffers the reference's caller owns. */
dprop_status dprop_release_cache(void);

/* Number of surfaces / volumes held by a detector (for callers sizing output). */
dprop_status dprop_detector_info(const dprop_detector* det, uint32_t* n_volumes,
                                 uint32_t* n_surfaces);

/* ------------------------------------------------------------- adjoint mode
 * dprop_propagate_adjoint and dprop_backward have no counterpart in the
 * reference.  They give reverse-mode derivatives of a loss L(b_1 .. b_K) of
 * the recorded bound parameters b_k of each track: dL/d(initial free
 * parameters) and dL/d(alignment) of the surfaces the records lie on.  The
 * factors of the chain are the surface-to-surface Jacobians the reference's
 * parameter transporter forms for its covariance transport
 * (core/include/detray/propagator/actors/parameter_updater.hpp:422-572), the
 * start-to-first-surface Jacobian and the derivative of the material
 * interaction's q/p kick.
 *
 * dprop_propagate_adjoint is dprop_propagate (plain kernel; launch->method and
 * use_graph are ignored) plus a tape of derivative data:
 *   tape->rec:  float [DPROP_TAPE_RECORD_FLOATS][max_records][n]
 *   tape->init: float [DPROP_TAPE_TRACK_FLOATS][n]
 * (device memory, written for every stored transported record and every
 * track with one).  Unlike dprop_propagate it restarts the transport
 * Jacobian at the first transported surface too, so the covariance it
 * records at the second transported surface follows the clean chain rather
 * than the reference's (which integrates that step's Jacobian from the track
 * start).  All other results are the same.  The results' rec_bound,
 * rec_barcode, rec_flags and n_records are required.
 *
 * dprop_backward runs the reverse sweep (one thread per track):
 *   grads->grad_bound[6]: float [max_records][n] (slot-major like rec_bound)
 *       dL/db_k; NULL entries are zero.
 *   grads->grad_free[8]: float [n] each, written: dL/d(x, y, z, t, tx, ty,
 *       tz, q/p) at the start; the direction part is tangent to the unit
 *       sphere (inputs are unit directions).  NULL entries are skipped.
 *   grads->grad_align: double [n_surfaces][6], ACCUMULATED (zero it first):
 *       dL/d(dt_x, dt_y, dt_z, w_x, w_y, w_z) of each planar or ring
 *       surface, a translation dt and a small rotation w (global axes) about
 *       the surface centre.  NULL: skipped.
 * The q/p row and time column of the Jacobians are identity (the reference's
 * convention), so time derivatives pass straight through.  Step sizes and
 * navigation decisions are constants of the derivative; the field map's
 * gradient enters through the position columns of the transport Jacobian
 * when cfg->use_field_gradient is set (the reference's with-gradient
 * Jacobian), and is left out otherwise (its default). */
#define DPROP_TAPE_RECORD_FLOATS 27u
#define DPROP_TAPE_TRACK_FLOATS 35u

typedef struct dprop_tape {
    void* rec;
    void* init;
} dprop_tape;

typedef struct dprop_gradients {
    const void* grad_bound[6];
    void* grad_free[8];
    double* grad_align;
} dprop_gradients;

dprop_status dprop_propagate_adjoint(const dprop_config* cfg,
                                     const dprop_launch* launch,
                                     const dprop_detector* det,
                                     const dprop_field* field,
                                     const dprop_tracks* tracks,
                                     const dprop_results* results,
                                     const dprop_tape* tape, uint64_t n_tracks,
                                     void* stream);

dprop_status dprop_backward(const dprop_config* cfg, const dprop_detector* det,
                            const dprop_tracks* tracks,
                            const dprop_results* results,
                            const dprop_tape* tape,
                            const dprop_gradients* grads, uint64_t n_tracks,
                            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DETRAY_B200_DPROP_H */
