/*
 * ncgpu.h - C ABI of the B200 engine for NcorpiON's mutual-interaction hot path.
 *
 * Plain C, no CUDA or torch types: every entry point takes host pointers,
 * sizes and PODs (the *_dev variants take device pointers as void* / double*),
 * and returns 0 (NCGPU_OK) or a negative NCGPU_E_* status.  The library owns a
 * single, device-resident body state between calls (single host thread,
 * single CUDA stream, not re-entrant), mirroring the reference's global state
 * (src/structure.c:62-115).
 *
 * Body records use the reference's `struct moonlet` layout
 * (src/structure.h:74-84): x, y, z, vx, vy, vz, mass, radius, all double.
 */
#ifndef NCGPU_H
#define NCGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define NCGPU_OK 0
#define NCGPU_E_ARG (-1)       /* bad argument (null pointer, size, mode)            */
#define NCGPU_E_CUDA (-2)      /* a CUDA runtime call failed                          */
#define NCGPU_E_CAPACITY (-3)  /* a device append buffer (pairs, events) overflowed   */
#define NCGPU_E_NMAX (-4)      /* a body append went past N_max (src/structure.c:860) */
#define NCGPU_E_STATE (-5)     /* ncgpu_init was not called / state not uploaded      */
#define NCGPU_E_TIMEOUT (-6)   /* a bounded device-side wait gave up                  */
#define NCGPU_E_UNSUPPORTED (-7) /* configuration outside the implemented hot path    */
#define NCGPU_E_FRAGMENT (-8)  /* fragmentation: a fragment slower than the escape
                                  velocity (the reference aborts, src/physics.c:818,934) */

/* Gravity arithmetic modes. */
#define NCGPU_GRAVITY_EXACT 0  /* FP64, the reference's per-body summation order and
                                  operation sequence: bit-identical to vector_field  */
#define NCGPU_GRAVITY_FP64 1   /* FP64, space-filling-curve tiles, one rsqrt per pair */
#define NCGPU_GRAVITY_MIXED 2  /* FP32 pair terms on tile-relative coordinates,
                                  near tiles in FP64, FP32 runs of 64 sources folded
                                  into FP64 sums */

/* Collision resolution types, numbered as collision_treatment's
   type_of_collision (src/physics.c:1043-1050). */
#define NCGPU_COLLISION_ELASTIC 0
#define NCGPU_COLLISION_INELASTIC 1
#define NCGPU_COLLISION_MERGER 2
#define NCGPU_COLLISION_FRAGMENTATION 3

struct ncgpu_body {          /* = struct moonlet (src/structure.h:74-84) */
      double x, y, z, vx, vy, vz, mass, radius;
};

struct ncgpu_pair {          /* = struct pair (src/structure.h, pairs[] of mesh()) */
      int fst, snd;
};

struct ncgpu_event {         /* one collision_treatment(a, b, type) call, in order */
      int a, b, type;
};

/* Mirror of the parameters.h macros that the hot path reads
   (src/parameters.h:66-119, 171-201, 283-309).  Each field is the macro's
   name with a par_ prefix, so this header can be included next to
   parameters.h, whose macros would otherwise rewrite the field names. */
struct ncgpu_params {
      double par_G;                      /* G                                        */
      double par_softening_parameter;    /* softening_parameter (x (R_k + R_p))      */
      int par_central_mass_bool;         /* central_mass_bool                        */
      int par_mutual_bool;               /* mutual_bool                              */
      int par_collision_bool;            /* collision_bool                           */
      int par_brute_force_bool;          /* brute_force_bool                         */
      int par_mesh_bool;                 /* mesh_bool                                */
      int par_collision_type;            /* NCGPU_COLLISION_*                        */
      double par_collision_parameter;    /* collision_parameter (inelastic f)        */
      int par_one_collision_only_bool;   /* one_collision_only_bool                  */
      int par_collision_cube_cells;      /* collision_cube_cells (mesh)              */
      double par_how_many_neighbours;    /* how_many_neighbours (mesh)               */
      double par_collision_cube_min;     /* collision_cube_min (mesh)                */
      int par_switch_to_brute_force;     /* switch_to_brute_force                    */
      int par_gravity_mode;              /* NCGPU_GRAVITY_*                          */
      double par_near_theta;             /* MIXED: tile pairs whose boxes are closer
                                        than near_theta x the larger box diagonal
                                        are summed in FP64 (default 0.15 if <= 0) */
      double par_disruption_threshold;   /* disruption_threshold (dump into the CM)  */
      double par_high_dumping_threshold; /* high_dumping_threshold (dump, unbound)   */
      int par_reduce_to_COM_bool;        /* reduce_to_COM_bool                       */
      /* fragmentation model, collision type NCGPU_COLLISION_FRAGMENTATION
         (src/parameters.h:297-307) */
      int par_N_tilde;                   /* N_tilde (<= NCGPU_MAX_N_TILDE)           */
      int par_pq_min_max[4];             /* pq_min_max {p_min, p_max, q_min, q_max};
                                            (p_max-p_min+1)(q_max-q_min+1) = N_tilde  */
      double par_mu_parameter;           /* mu_parameter                             */
      double par_nu_parameter;           /* nu_parameter                             */
      double par_C1_parameter;           /* C1_parameter                             */
      double par_k_parameter;            /* k_parameter                              */
      double par_merging_threshold;      /* merging_threshold                        */
      double par_fragment_threshold;     /* fragment_threshold                       */
      /* Mesh driver only, no reference counterpart: 1 replaces the mesh gravity
         (pairs[] + the three largest bodies) by the brute-force field of
         par_gravity_mode over every body, keeping the mesh collision search. */
      int par_mesh_brute_gravity;
      /* the central body's symmetrical equatorial bulge (src/physics.c:149-160),
         which needs the central mass.  par_J2 is parameters.h's J2_value: a
         nonzero value is the J2; 0 selects the fluid-body
         J2 = 0.5*SideralOmega*SideralOmega*R_unit^3/(G*M), re-evaluated from the
         current central mass M at every force evaluation (src/structure.c:507,
         src/rk4.c:459-463; M only changes in end_of_timestep).
         par_sideral_omega is SideralOmega = 2*pi/Tearth. */
      int par_J2_bool;
      double par_J2;
      double par_R_unit;
      double par_sideral_omega;
      /* tides raised on the central body, constant time lag model (tides,
         src/physics.c:496-542, called from kick, src/rk4.c:88-90): k2, Delta_t
         and dimensionless_moi (src/parameters.h:143-145).  Tides change the
         central body's sideral rotation, which is then device state
         (ncgpu_get_sideral_omega).  Needs the central mass. */
      int par_central_tides_bool;
      double par_k2;
      double par_Delta_t;
      double par_dimensionless_moi;
};
#define NCGPU_MAX_N_TILDE 64

/* Fills *p with the reference's default values for the fields above
   (fragmentation constants: N_tilde 15 on {-1,3,-1,1}, mu 0.55, nu 0.4,
   C1 1.5, k 0.2, merging 2e-4, fragment 1.5e-8, src/parameters.h:297-307)
   and G = 39.478..., softening 0, central mass on, mutual on, ... */
void ncgpu_default_params(struct ncgpu_params *p);

/* Allocates device state for n_max body slots (N_max, src/parameters.h:171)
   and copies the parameters.  Replaces array_initialization's allocations
   (src/structure.c:553-647). */
int ncgpu_init(int n_max, const struct ncgpu_params *params);
void ncgpu_finalize(void);
/* Replaces the parameters of an initialised library (no reallocation). */
int ncgpu_set_params(const struct ncgpu_params *params);
const char *ncgpu_strerror(int status);
/* Last CUDA error string recorded by the library (for NCGPU_E_CUDA). */
const char *ncgpu_last_error(void);

/* ---- stateless force evaluation ------------------------------------------ */

/* vector_field (src/physics.c:63-441), brute-force branch with the central
   mass term: for every slot k <= largest_id with exists[k] != 0, writes the
   acceleration of body k into bodies[k].vx, vy, vz (the reference stores
   accelerations in the velocity fields, src/physics.c:264-266) and the central
   mass back-reaction into cm_acc[3] (CM_acc, src/physics.c:137-139).  Host
   buffers; copies in and out on the library stream.  The records come back
   whole in one copy: every byte other than those velocity fields is the
   caller's own (on an error status the velocity fields may be overwritten). */
int ncgpu_vector_field(struct ncgpu_body *bodies, const int *exists, int largest_id,
                       const struct ncgpu_body *cm, double *cm_acc, int gravity_mode);

/* Same computation on device-resident buffers: d_bodies holds 8 doubles per
   slot (struct moonlet layout), d_exists one int per slot, d_acc receives
   3 doubles per slot (zero for empty slots), d_cm_acc 3 doubles.  cm points to
   host memory.  stream is a cudaStream_t (NULL = the library stream).  The
   call is asynchronous on that stream: a device wait that gave up (or another
   device-side error) is reported by ncgpu_check_error, or by the next call
   that waits for the library stream. */
int ncgpu_vector_field_dev(const double *d_bodies, const int *d_exists, int largest_id,
                           const struct ncgpu_body *cm, double *d_acc, double *d_cm_acc,
                           int gravity_mode, void *stream);

/* One part of the same field, for runs that split the targets over several
   GPUs (one process per GPU; the parts exchange through an all-reduce sum):
   only the targets of part `part` of `nparts` get their acceleration -- the
   part-th slice of the existing bodies in slot order (exact mode), or of the
   Morton-ordered 128-body target blocks (FP64 / mixed) -- and every other row
   of d_acc receives -0.0 (+0.0 for empty slots from part 0), the identity of
   the sum, so that the element-wise sum of the parts' d_acc is the full field
   bit for bit.  d_cm_acc receives the full CM_acc in every part.
   ncgpu_vector_field_dev is part 0 of 1.  (No reference counterpart: the
   reference is single-threaded; the sum of the parts is vector_field's.) */
int ncgpu_vector_field_part(const double *d_bodies, const int *d_exists, int largest_id,
                            const struct ncgpu_body *cm, int part, int nparts, double *d_acc,
                            double *d_cm_acc, int gravity_mode, void *stream);

/* Waits for `stream` (NULL = the library stream) and for the library stream,
   then returns and clears the status that device kernels recorded since the
   last check: NCGPU_E_TIMEOUT for a bounded device wait that gave up,
   NCGPU_E_CAPACITY / NCGPU_E_NMAX for a device-side overflow, NCGPU_OK when
   nothing was recorded.  (No reference counterpart: the reference has no
   asynchronous calls.) */
int ncgpu_check_error(void *stream);

/* Allocation-free variant of ncgpu_vector_field_dev in the EXACT mode.  It has
   no counterpart in the reference: it exists for callers that cannot allocate
   device memory when they evaluate forces (a host whose device memory belongs to
   its own pool allocator, an integration loop that forbids allocation once it
   runs).  It needs no ncgpu_init and calls no cudaMalloc or cudaFree: its scratch
   is a fixed file-scope device array of ncgpu_noalloc_scratch_bytes() bytes,
   held by every GPU that the library's device code is loaded on, sized for at most
   NCGPU_NOALLOC_MAX_SLOTS body slots (largest_id + 1 larger than that returns
   NCGPU_E_CAPACITY).  CUDA loads device code lazily by default, so the array
   and the kernels reach a device at the first call on it: that call is the
   set-up (it loads them and looks up the array's device address with
   cudaGetSymbolAddress).  Make one call on each device before the host's pool
   allocator takes the device's memory and before any stream capture, or run
   with CUDA_MODULE_LOADING=EAGER; after cudaDeviceReset do not call it again.
   All calls share the array and it keeps the last call's contents: calls that
   overlap on the GPU race.  params supplies G, softening_parameter,
   central_mass_bool and the central body's J2 (par_J2_bool, par_J2, par_R_unit,
   par_sideral_omega for the fluid-body J2 when par_J2 is 0; J2 without a
   central mass returns NCGPU_E_ARG); the other arguments are those of
   ncgpu_vector_field_dev (stream may be NULL: the default stream).  The call
   waits for its stream and returns NCGPU_E_TIMEOUT if a device wait gave up. */
#define NCGPU_NOALLOC_MAX_SLOTS 65536
int ncgpu_vector_field_static(const double *d_bodies, const int *d_exists, int largest_id,
                              const struct ncgpu_body *cm, const struct ncgpu_params *params,
                              double *d_acc, double *d_cm_acc, void *stream);
unsigned long ncgpu_noalloc_scratch_bytes(void);

/* Number of kernel launches issued by the last API call. */
int ncgpu_last_launch_count(void);
/* The library's CUDA stream (a cudaStream_t), for callers that time or order
   work against it; NULL before ncgpu_init. */
void *ncgpu_stream(void);
/* Device time (CUDA events on the launching stream) of the dominant kernel of
   the last gravity evaluation (the pair-sum kernel), in milliseconds. */
int ncgpu_last_kernel_ms(double *ms);

/* Page-locks a host buffer (e.g. the reference's moonlets array) so the
   library's host<->device copies of it run at full bus speed. */
int ncgpu_host_register(void *ptr, unsigned long bytes);
int ncgpu_host_unregister(void *ptr);

/* Diagnostic: measures this GPU's FP32 FFMA throughput with a dependent-chain
   kernel (2 flops per FFMA) and returns it in *tflops; used as the roofline
   denominator of the FP32 gravity kernel. */
int ncgpu_probe_fp32_peak(double *tflops);
/* Diagnostic (no reference counterpart): measured FP32 rates of this GPU,
   from independent dependency chains: scalar FFMA and packed f32x2 FMA in
   TFLOP/s (2 flops per FMA lane), and rsqrt.approx.f32 in Gop/s. */
int ncgpu_probe_fp32_rates(double *ffma_tflops, double *ffma2_tflops, double *rsqrt_gops);
/* Diagnostic (no reference counterpart): a kernel waits on a barrier that
   nothing completes, giving up after `probes` failed probes (1 .. 2^20, the
   library's limit for every device wait), as every bounded wait here does.
   Returns NCGPU_E_TIMEOUT with the cycles one failed probe took; the library
   stays usable.  Tests the timeout path without hanging a GPU. */
int ncgpu_probe_wait_timeout(int probes, double *cycles_per_probe);

/* Diagnostic: out[i] = x[i]^(1.0/3.0), correctly rounded, as the device
   merger computes the merged radius (src/physics.c:684). */
int ncgpu_probe_pow_third(const double *x, double *out, int n);
/* a[i] / b[i] with the correctly rounded division of the tides' recurrence
   (reciprocal and two residual corrections), for tests.  Host buffers. */
int ncgpu_probe_div(const double *a, const double *b, double *out, int n);
/* Diagnostic: out[c] = s0[c] + x[c*n] + x[c*n + 1] + ... + x[c*n + n-1] for the
   `chains` chains, added in that order with round-to-nearest after every
   addition (the plain loop's bits), by the device routines that form the
   reference-order sums here: the one that takes whole runs of terms within a
   binade (runs != 0; display()'s total mass of 65,536 bodies or more) or the
   staged one-add-at-a-time loop (runs == 0; every other such sum).  Host
   buffers. */
int ncgpu_probe_seq_sum(const double *x, long n, const double *s0, double *out, int chains, int runs);

/* ---- device-resident integrator state ------------------------------------ */

/* Uploads slots 0..largest_id (bodies + exists) and the central mass. */
int ncgpu_upload(const struct ncgpu_body *bodies, const int *exists, int largest_id,
                 const struct ncgpu_body *cm);
/* Downloads slots 0..*largest_id into host arrays of at least n_max slots. */
int ncgpu_download(struct ncgpu_body *bodies, int *exists, int *largest_id,
                   struct ncgpu_body *cm);
/* timestep global (src/structure.c, used by kick/drift/closest_approach). */
int ncgpu_set_timestep(double dt);

/* kick (src/rk4.c:68-106) with F = vector_field in the configured gravity
   mode: v += timestep * a for existing bodies, CM.v += timestep * CM_acc. */
int ncgpu_kick(void);
/* drift (src/rk4.c:109-127): x += timestep * v, CM too. */
int ncgpu_drift(void);

/* brute_force (src/collision.c:425-456): every pair i < j in the reference's
   sweep order, FP64 closest_approach predicate, in-place resolution by
   collision_treatment (src/physics.c:1043) with the configured type.
   *n_events receives the number of collision_treatment calls. */
int ncgpu_collide_brute(int *n_events);

/* Total energy of the device state (no reference counterpart; the reference
   has no energy output): out[0] = E, out[1] = kinetic (bodies and central
   body), out[2] = central-body potential, out[3] = mutual potential with the
   force's softening sqrt(r^2 + (softening_parameter (R_k + R_p))^2).  FP64,
   O(N^2), deterministic; for energy-drift diagnostics. */
int ncgpu_energy(double *out);
/* The central body's sideral rotation SideralOmega (src/structure.c:110), part
   of the device state: ncgpu_init sets it to par_sideral_omega, the tides of
   every kick change it (src/physics.c:539), and the fluid-body J2 of the
   state-based kicks is evaluated from it.  The stateless vector_field entry
   points use par_sideral_omega. */
int ncgpu_get_sideral_omega(double *omega);
/* The J2 in force for the state's kicks (J2_value, or the fluid-body J2 of the
   last upload or end of step, src/rk4.c:459-463) and, in j2_before (may be
   NULL), the one before the last end of step's update -- the value
   end_of_timestep's printout still sees (src/rk4.c:225-333 precede the
   update).  0 without J2. */
int ncgpu_get_j2(double *j2, double *j2_before);
int ncgpu_set_sideral_omega(double omega);
/* Output staging (display(), src/display.c:239-451, at the drivers' output
   steps).  ncgpu_snapshot_begin copies the bodies' fields and the central body
   and makes the copy the state: until ncgpu_snapshot_end every entry point
   (drift, kick, three_largest, mesh, the two calls below) works on the copy,
   while exists[], the free slots and largest_id stay shared with the original,
   as the reference's globals are shared between its body array and the copy it
   prints (src/rk4.c:740-757, 881-890).  ncgpu_snapshot_end makes the original
   the state again; SideralOmega keeps the copy's value (one global in the
   reference). */
int ncgpu_snapshot_begin(void);
int ncgpu_snapshot_end(void);
/* The cartesian files' text of this output for the current state (display()
   with write_cartesian_bool): x, y, z, vx, vy, vz (the central body first when
   par_central_mass_bool), mass, radius, each value as "%.14lf " (the exact
   decimal of the double rounded to 14 digits, ties to even, as glibc prints it)
   over the existing bodies in slot order.  The 8 files' texts are concatenated
   in `text` (no newlines; display() ends each line with one) and lens[8]
   receives their byte counts.  cap >= ncgpu_format_cartesian_cap() always
   suffices.  NCGPU_E_UNSUPPORTED when a value exceeds 1.7e24 in magnitude
   (the caller prints that output itself).  It also starts the statistics of
   ncgpu_output_stats on a second stream, so that a call of that function
   right after this one (as display() makes them) finds them computed. */
int ncgpu_format_cartesian(char *text, unsigned long cap, unsigned long *lens);
unsigned long ncgpu_format_cartesian_cap(void);
/* The elliptic files of this output (display() with write_elliptic_bool,
   src/display.c:340-347: cart2ell, src/structure.c:172-284, of every existing
   body in slot order with mu + G*m), in two calls around the caller's libm.
   ncgpu_elliptic_begin computes on the device, in the reference's operation
   order, a, k, h, q, p and the two arguments of the mean longitude's atan2
   (src/structure.c:268-271): yx[2j], yx[2j+1] = sinF, cosF of the j-th
   existing body (0, 0 where the longitude is 0: R or V2 zero), yx_cap >= 2 *
   *n_bodies.  Bodies that cart2ell takes out of that branch -- hyperbolic
   (src/structure.c:274-279), printing its (k, h) warning (src/structure.c:
   253-255) or giving a NaN -- are listed: host_idx their slots (ascending),
   host_rec their records; the caller converts them with its cart2ell, which
   prints the warnings as display() does.  NCGPU_E_CAPACITY when *n_host >
   host_cap.  mu is display()'s mu (G times the central mass or M_unit); the
   central body, J2_bool, J2 (the one in force), R_unit and G come from the
   state and the parameters.
   ncgpu_format_elliptic takes F[j] = atan2(yx[2j], yx[2j+1]) for every body
   (entries of listed bodies are ignored) and host_alkhqp[6k .. 6k+5], cart2ell's
   alkhqp of listed body k, and returns the texts of a, lambda, k, h, q, p (then
   mass and radius when mass_radius) like ncgpu_format_cartesian, lens[6] or
   lens[8], with the same capacity bound and NCGPU_E_UNSUPPORTED rule.  After it,
   ncgpu_elliptic_values copies the elements and the bodies' masses and radii
   (8 blocks of *n_bodies doubles, cap >= 8 * *n_bodies) for a caller that
   prints them itself.  No state change may come between the calls. */
int ncgpu_elliptic_begin(double mu, double *yx, unsigned long yx_cap, int *n_bodies, int *host_idx,
                         struct ncgpu_body *host_rec, int host_cap, int *n_host);
int ncgpu_format_elliptic(const double *F, const double *host_alkhqp, int n_host, int mass_radius, char *text,
                          unsigned long cap, unsigned long *lens);
int ncgpu_elliptic_values(double *values, unsigned long cap);
/* F[j] = atan2(yx[2j], yx[2j+1]) for j < n with the C library's atan2 (the
   function cart2ell calls; glibc's is not correctly rounded in every case, so
   the files' bytes need that very function), on up to 16 host threads: the
   loop between ncgpu_elliptic_begin and ncgpu_format_elliptic, for callers
   that have none of their own. */
int ncgpu_host_atan2(const double *yx, double *F, long n);
/* display()'s statistics of the current state (src/display.c:303-379):
   stats[0] the total mass of the bodies summed in slot order, stats[1..2] and
   idx[0..1] the masses M1, M2 and slots of the two most massive bodies as its
   loop picks them (0 when absent), two[0..1] those slots' records, cm the
   central body.  Computed here, or taken from the preceding call when that was
   ncgpu_format_cartesian on the same state. */
int ncgpu_output_stats(double *stats, int *idx, struct ncgpu_body *cm, struct ncgpu_body *two);
/* The barycentre end_of_timestep prints at a progress step (src/rk4.c:202-222,
   333): zeros right after an ncgpu_end_of_timestep that reduced the barycentre
   (the reference zeroes the vector it subtracted), otherwise the state's
   total_momentum (src/structure.c:1193-1227), exact sums in slot order. */
int ncgpu_total_momentum(double *com);
/* largest_id of the device state, and (before_tidy, may be NULL) its value at
   the start of the last ncgpu_end_of_timestep, before tidy_up -- the one
   end_of_timestep prints (src/rk4.c:235-240). */
int ncgpu_get_largest_id(int *largest_id, int *before_tidy);
/* Outcomes of the fragmentation model since the last upload, in the order of
   merger_count, super_catastrophic_count, half_fragmentation_count and
   full_fragmentation_count (src/structure.h:148-151). */
int ncgpu_fragment_counts(int *counts);
/* The events of the last sweep, in resolution order: (a, b, type) as passed to
   collision_treatment, and optionally 8 doubles per event for the collision
   output file: time_until_collision, m_A, m_B, R_A, R_B (A the heavier body,
   values before the collision), DeltaV and dr.dv (src/physics.c:612-617). */
int ncgpu_get_events(struct ncgpu_event *events, double *records, int cap, int *n_events);

/* end_of_timestep (src/rk4.c:130-404), hot-path part: bodies inside
   disruption_threshold merge into the central mass, bodies beyond
   high_dumping_threshold are removed (then the barycentre is reduced when
   reduce_to_COM_bool), did_collide is reset when collisions are limited, and
   the body array is compacted by tidy_up when fewer than 9/10 of
   largest_id slots are used.  *how_many_moonlets receives the body count. */
int ncgpu_end_of_timestep(int *how_many_moonlets);

/* ---- mesh ------------------------------------------------------------------ */

/* three_largest_moonlets + three_largest_three_first (src/structure.c:914-1063):
   the three largest bodies (by radius) moved to slots 0, 1, 2; idx receives
   three_largest_indexes before the moves (may be NULL). */
int ncgpu_three_largest(int *idx);

/* One pass of the mesh algorithm with mesh size gam (collision_cube =
   gam * collision_cube_cells).  with_collisions = 1: mesh()
   (src/collision.c:324-417): bodies with R <= gam, FP64 closest_approach on
   every popped pair in the reference's pop order, collisions resolved in
   place; 0: get_neighbours_mesh() (src/physics.c:1094): every body, no test.
   Outputs: the length of pairs[] (how_many_pairs), the number of events and
   total_neighbours.  Bodies larger than gam are not supported by the
   parallel pass (NCGPU_E_UNSUPPORTED). The pass's cell table stays valid for
   the next kick (mesh gravity) until end_of_timestep or ncgpu_mesh_reset. */
int ncgpu_mesh(double gam, int with_collisions, int *n_pairs, int *n_events, long *total_neighbours);
/* pairs[] of the last pass in the reference's order (struct pair). */
int ncgpu_get_pairs(struct ncgpu_pair *pairs, int cap, int *n_pairs);
/* Clears the cell table of the last pass (the hash reset of src/rk4.c:361). */
int ncgpu_mesh_reset(void);
/* force_naive_bool: 1 switches kicks and collisions to the brute-force path
   (set by the host when N < switch_to_brute_force, src/rk4.c:388-393). */
int ncgpu_set_force_naive(int on);

/* One iteration of integration_mesh's loop (src/rk4.c:760-790): three largest
   to slots 0-2, mesh() (or brute force when force_naive), drift, kick with
   mesh gravity, end_of_timestep.  The host owns gamma and updates it from
   total_neighbours with the reference's formula (src/rk4.c:367-372). */
int ncgpu_step_mesh(double gam, int *how_many_moonlets, long *total_neighbours);

/* One iteration of integration_brute_force_SABA1's loop (src/rk4.c:906-921):
   kick, brute_force collisions (when collision_bool), drift, end_of_timestep. */
int ncgpu_step_brute_force(int *how_many_moonlets);

/* ---- differentiable leapfrog (no reference counterpart) ------------------ */

/* Host arrays, bodies as (n, 3) row-major triples. */
struct ncgpu_leapfrog_args {
      int n;                       /* bodies (all existing)                      */
      const double *x0, *v0;       /* initial positions / velocities, 3n each     */
      const double *m, *R;         /* masses, radii (softening), n each           */
      const double *cm;            /* central mass record, 8 doubles              */
      double dt;                   /* timestep                                    */
      int nsteps;                  /* leapfrog steps                              */
      int checkpoint;              /* steps between stored states (default 32)    */
      double *x_final, *v_final;   /* outputs (3n each, may be NULL)              */
      const double *adj_x_final;   /* dL/dx_final, 3n (ncgpu_leapfrog_vjp)        */
      double *grad_x0, *grad_v0;   /* dL/dx0, dL/dv0, 3n each (ncgpu_leapfrog_vjp) */
      double *grad_m;              /* dL/dm, n (ncgpu_leapfrog_vjp)                */
      const double *tan_x0, *tan_v0, *tan_m;  /* input tangents (ncgpu_leapfrog_jvp)  */
      double *tan_x_final;         /* output tangent of x_final, 3n (ncgpu_leapfrog_jvp) */
};

/* The brute-force integrator without collisions (src/rk4.c:873-936): half
   drift, nsteps x (kick, drift), half back-drift of the output, the central
   mass integrated as a body.  FP64 pair sums, one rsqrt per pair (par_gravity_mode
   MIXED: far tile pairs in FP32).  The three calls share one device buffer, grown
   when a call needs more and kept until ncgpu_finalize. */
int ncgpu_leapfrog(const struct ncgpu_leapfrog_args *args);

/* Reverse mode through ncgpu_leapfrog: given dL/dx_final returns dL/dx0,
   dL/dv0 and dL/dm.  States are stored every `checkpoint` steps and each
   segment is recomputed, so memory is O(n (nsteps/checkpoint + checkpoint)). */
int ncgpu_leapfrog_vjp(const struct ncgpu_leapfrog_args *args);

/* Forward mode (tangent-linear) through ncgpu_leapfrog: the directional
   derivative of x_final along (tan_x0, tan_v0, tan_m).  Exact to rounding, it
   checks the adjoint through <w, J d> = <J^T w, d> where finite differences of
   tiny masses drown in roundoff. */
int ncgpu_leapfrog_jvp(const struct ncgpu_leapfrog_args *args);

#ifdef __cplusplus
}
#endif
#endif /* NCGPU_H */
