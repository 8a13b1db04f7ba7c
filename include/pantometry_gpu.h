/*
 * pantometry_gpu.h — the C ABI of the B200-native stepping path.
 *
 * One library, libpantometry_b200.so, holds sm_100a CUDA kernels and a C++ host runtime for
 * six of pantometry's `Domain` implementations, and an ensemble of many `Solid3D` blocks:
 *
 *   pm_heat    ~ Solid3D  (crates/pantometry-thermal/src/solid.rs)
 *   pm_hall    ~ Hall     (crates/pantometry-acoustic/src/hall.rs)
 *   pm_room    ~ Room     (crates/pantometry-acoustic/src/room.rs)
 *   pm_tube    ~ Tube     (crates/pantometry-acoustic/src/lib.rs:107-560)
 *   pm_bar     ~ Bar1D    (crates/pantometry-thermal/src/lib.rs:425-660)
 *   pm_cavity  ~ Cavity   (crates/pantometry-em/src/cavity.rs)
 *
 * Each handle is the device-side state of one domain and answers the calls a `Domain` answers
 * (crates/pantometry-core/src/sim.rs:77-252): step, ledger, max_stable_dt, checkpoint, restore.
 * Every step computes the domain's energy ledger on the device in FP64 with a fixed-order
 * reduction tree (run-to-run reproducible), and can audit it against the previous step the way
 * `Simulation::advance` does (sim.rs:947-965, conserved.rs:323-363) without a host round trip.
 *
 * Two arithmetic forms per domain (pm_precision):
 *   PM_PLAIN_F64   IEEE f64, no FMA contraction, the reference's operand order: bit-exact with
 *                  the reference cell by cell.
 *   PM_FIELDS_F32  fields stored and updated in f32 (heat stores T − T0); ledgers, audits and
 *                  the running books stay in f64.
 *
 * Conventions: plain pointers and sizes, host memory unless a name says `device`. Every call
 * returns a pm_status; nothing calls exit() or abort(). pm_last_error() gives the message of
 * the last failing call on the calling thread. There is no CPU fallback: without a CUDA device
 * pm_*_create returns PM_NO_DEVICE.
 */
#ifndef PANTOMETRY_GPU_H
#define PANTOMETRY_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Replaces `Result<(), Violation>` (sim.rs:77-252) and
 * `Unavailable{NoAdapter, NoDevice, NotConducting}` (runtime/gpu/src/lib.rs:99-106). */
typedef enum pm_status {
    PM_OK = 0,
    PM_NO_DEVICE = 1,      /* no CUDA device, or the library's kernels cannot run on it */
    PM_UNSUPPORTED = 2,    /* a feature the kernels do not implement (e.g. phase change) */
    PM_VIOLATION = 3,      /* a step was refused or an audit failed; the pm_violation is filled */
    PM_DEVICE_TIMEOUT = 4, /* a bounded wait inside a kernel ran out (the TMA-staged kernels wait on
                            * their own copies); the call stopped, and the fields of the step that
                            * gave up are incomplete: restore a checkpoint before going on */
    PM_BAD_ARG = 5,
    PM_CUDA_ERROR = 6,
    PM_OUT_OF_MEMORY = 7
} pm_status;

typedef enum pm_precision { PM_PLAIN_F64 = 0, PM_FIELDS_F32 = 1 } pm_precision;

/* `Violation` (crates/pantometry-core/src/conserved.rs:128-143), plus the step it happened on. */
typedef struct pm_violation {
    char quantity[32];
    char site[96];
    double before;
    double after;
    double scale;
    double tolerance;
    long long step; /* 1-based index, within the failing call, of the step that failed */
} pm_violation;

/* The "energy" `Entry` of a `Ledger` (conserved.rs:37-124): its total and scale, and the
 * contributions that `Ledger::with` added, in order:
 *   heat:   stored, lost, -supplied                          (solid.rs:1904-1927)
 *   hall:   invariant + offset (- source injection)          (hall.rs:532-534)
 *   cavity: invariant, dissipated (, -source work)           (cavity.rs:1520-1524) */
typedef struct pm_ledger {
    double total;
    double scale;
    double parts[4];
    int n_parts;
    long long steps; /* steps taken since the state was last uploaded or released */
} pm_ledger;

const char* pm_status_string(pm_status status);
const char* pm_last_error(void);
pm_status pm_device_count(int* count);
const char* pm_version(void);

/* ==================================== Solid3D ====================================== */

typedef struct pm_heat pm_heat;

/* `Substance` with its `ThermalProps` (crates/pantometry-core/src/substance.rs:43-92, 108-123).
 * thermal == 0 is `thermal: None`, which leaves the block with no diffusivity. */
typedef struct pm_substance {
    double density;       /* kg/m^3 */
    double conductivity;  /* W/m/K */
    double specific_heat; /* J/kg/K */
    double emissivity;
    int thermal;
} pm_substance;

typedef struct pm_heat_desc {
    const char* name;
    int nx, ny, nz;
    double dx;
    pm_substance substance;
    double initial_kelvin; /* also the enthalpy reference stored heat is measured from */
    int precision;         /* pm_precision */
    int device;
} pm_heat_desc;

/* Solid3D::new (solid.rs:377-421). */
pm_status pm_heat_create(const pm_heat_desc* desc, pm_heat** out);
/* Solid3D::fill (solid.rs:519-543): cells with mask[c] != 0 take `substance`. */
pm_status pm_heat_fill(pm_heat* h, const pm_substance* substance, const uint8_t* mask, size_t n);
/* Solid3D::losing_from (solid.rs:1039-1043). face: 0..5 = XMin, XMax, YMin, YMax, ZMin, ZMax.
 * `area` is the whole face's area; convection may be +inf (a Dirichlet face). */
pm_status pm_heat_losing_from(pm_heat* h, int face, double ambient_kelvin,
                              double convection_w_per_m2_k, double area);
/* Solid3D::empty (solid.rs:986-1005): cells with mask[c] != 0 become void. A void cell holds no
 * heat, conducts nothing, takes no share of absorbed heat and generates nothing; its value in the
 * downloaded field is a placeholder that never changes (solid.rs:1324-1335 reads it as NaN). Two
 * solid cells facing each other along a grid line across a run of void radiate to each other,
 * σA(T1^4 - T2^4)/(1/e1 + 1/e2 - 1) (solid.rs:786-838, 1866-1878); the limit then follows the
 * state, and a block with such gaps steps on the plain f64 form only. */
pm_status pm_heat_empty(pm_heat* h, const uint8_t* mask, size_t n);
/* Solid3D::dissipating (solid.rs:1045-1085): `watts` in total, spread evenly over the solid cells
 * with mask[c] != 0, replacing what they generated before; selecting no solid cell does nothing. */
pm_status pm_heat_dissipating(pm_heat* h, double watts, const uint8_t* mask, size_t n);
/* Solid3D::generated_power and generated_energy (solid.rs:1118-1126); either may be NULL. */
pm_status pm_heat_generated(pm_heat* h, double* watts, double* joules);
/* The gap pairs (first cell, second cell, coefficient in W/K^4) in the order the step applies
 * them; *count is the number of pairs, of which the first `capacity` are written. */
pm_status pm_heat_gaps(pm_heat* h, long long* a, long long* b, double* coefficient, size_t capacity,
                       size_t* count);
/* Solid3D::set_temperature over every cell (solid.rs:1346-1361), kelvin, index x + nx(y + ny z). */
pm_status pm_heat_upload(pm_heat* h, const double* kelvin, size_t n);
pm_status pm_heat_download(pm_heat* h, double* kelvin, size_t n);
/* Solid3D as a field (solid.rs:2028-2104): kelvin, trilinear between cell centres, clamped at the
 * faces, NaN in a void cell, the weights renormalised over the solid corners.
 * scene::capture's sampling (crates/pantometry-scene/src/lib.rs:347-420), run on the device over the
 * resident field: `samples[0] * samples[1] * samples[2]` points from `lo` to `hi` (metres, the
 * domain's own coordinates), x fastest, i / (n - 1) of the way along an axis of n > 1 samples and
 * the middle of an axis of one; `out` (host, n values) receives `ScalarField::at` at each point. */
pm_status pm_heat_sample(pm_heat* h, const double lo[3], const double hi[3], const int samples[3], double* out,
                         size_t n);
/* Domain::max_stable_dt (solid.rs:1709-1715). */
pm_status pm_heat_max_stable_dt(pm_heat* h, double* seconds);
/* Relative tolerance of the per-step audit (`Simulation::advance`, sim.rs:947-965, and
 * `attribute`, sim.rs:1169-1223). Negative disables it, leaving plain `Domain::step`. */
pm_status pm_heat_set_tolerance(pm_heat* h, double tolerance);
/* `nsteps` calls of Domain::step (solid.rs:1717-1901), each followed by the ledger and, when
 * enabled, the audit. Stops at the first violation (PM_VIOLATION, *out filled). */
pm_status pm_heat_step(pm_heat* h, double dt, long long nsteps, pm_violation* out);
/* Domain::ledger (solid.rs:1904-1927), as of the last step. */
pm_status pm_heat_ledger(pm_heat* h, pm_ledger* out);
/* Placeless heat off the bus (solid.rs:1752-1765): held until the next pm_heat_step, whose first
 * step takes it after its stability refusal (checked against the state before the rise) as a
 * uniform rise over the solid cells. A refused step leaves it held. */
pm_status pm_heat_absorb(pm_heat* h, double joules);
/* Domain::checkpoint / restore (solid.rs:1935-1950). */
pm_status pm_heat_checkpoint(pm_heat* h);
pm_status pm_heat_restore(pm_heat* h);
/* No counterpart in the reference. The kernel a call of pm_heat_step for `nsteps` steps would run
 * on the present block (its name, at most cap - 1 bytes and a terminating 0, into `name`) and how
 * many launches of it the call makes: one a step, or one per 1024 steps for the many-step
 * cooperative kernels of small uniform blocks. Nothing runs. */
pm_status pm_heat_step_kernel(pm_heat* h, long long nsteps, char* name, int cap, long long* launches);
/* Cells of a row per thread (no reference counterpart: a launch shape, like the ensemble's brick
 * shape). The default is the precision's widest form where the block is one material and its rows
 * allow: in plain f64, 4 adjacent cells per thread on rows of a multiple of 4 cells, else 2 on rows
 * of an even number; in FP32, 4 on rows of a multiple of 4. 1 takes one cell per thread; plain f64
 * also takes 2 or 4, FP32 4. The fields are the same bit for bit either way. */
pm_status pm_heat_set_cells_per_thread(pm_heat* h, int cells);
/* Run subsequent work on `stream` (a cudaStream_t); NULL restores the handle's own stream. */
/* No counterpart in the reference. Small uniform blocks (up to 2^22 cells, rows of an even number of
 * cells in plain f64 or a multiple of 4 in FP32, films that do not radiate) take many steps of one
 * call in one cooperative launch, one grid-wide wait per step. Each wait is bounded: `polls` looks at the
 * arrivals, each a few hundred ns apart (default 2^24, over a second); a wait that runs out stops the
 * call with PM_DEVICE_TIMEOUT and leaves the
 * fields of the step in progress incomplete. 0 makes every wait that is not already over give up at
 * once, which exercises that path without a fault. */
pm_status pm_heat_set_wait_budget(pm_heat* h, unsigned polls);
pm_status pm_heat_set_stream(pm_heat* h, void* stream);
void pm_heat_destroy(pm_heat* h);

/* ===================================== Hall ========================================= */

typedef struct pm_hall pm_hall;

typedef struct pm_hall_desc {
    const char* name;
    double width, height, depth; /* metres */
    int across;                  /* nodes along the width */
    double speed;                /* m/s */
    double density;              /* kg/m^3 */
    int precision;               /* pm_precision */
    int device;
} pm_hall_desc;

/* Hall::new (hall.rs:99-134). */
pm_status pm_hall_create(const pm_hall_desc* desc, pm_hall** out);
pm_status pm_hall_nodes(pm_hall* h, int* nx, int* ny, int* nz, double* dx);
/* Hall::released_from (hall.rs:166-184) with the profile sampled at the nodes. */
pm_status pm_hall_release(pm_hall* h, const double* pressure, size_t n);
/* Extension (not in the reference): a soft point source adding wave[s] Pa at `node` after the
 * pressure update of step s (s counted from the release); its work is kept in the ledger. */
pm_status pm_hall_set_source(pm_hall* h, long long node, const double* wave, size_t n);
/* Extension (not in the reference): a piecewise-constant sound speed over cubic blocks of
 * `block` nodes per side, speeds[b] for block index bx + nbx(by + nby bz). The step limit
 * follows the fastest block. */
pm_status pm_hall_set_speed_blocks(pm_hall* h, int block, const double* speeds, size_t n);
pm_status pm_hall_max_stable_dt(pm_hall* h, double* seconds);
pm_status pm_hall_set_tolerance(pm_hall* h, double tolerance);
/* `nsteps` calls of Domain::step (hall.rs:408-530), ledger and audit as for pm_heat_step. */
pm_status pm_hall_step(pm_hall* h, double dt, long long nsteps, pm_violation* out);
pm_status pm_hall_ledger(pm_hall* h, pm_ledger* out);
/* Any pointer may be NULL. p_prev is `pressure_prev`. */
pm_status pm_hall_download(pm_hall* h, double* p, double* p_prev, double* vx, double* vy, double* vz);
/* Hall as a field (hall.rs:585-613): pascals, trilinear between nodes, clamped at the surfaces.
 * scene::capture's sampling (crates/pantometry-scene/src/lib.rs:347-420), run on the device over the
 * resident field: `samples[0] * samples[1] * samples[2]` points from `lo` to `hi` (metres, the
 * domain's own coordinates), x fastest, i / (n - 1) of the way along an axis of n > 1 samples and
 * the middle of an axis of one; `out` (host, n values) receives `ScalarField::at` at each point. */
pm_status pm_hall_sample(pm_hall* h, const double lo[3], const double hi[3], const int samples[3], double* out,
                         size_t n);
pm_status pm_hall_checkpoint(pm_hall* h);
pm_status pm_hall_restore(pm_hall* h);
/* No counterpart in the reference. FP32 halls on the TMA-staged kernel (x extent a multiple of 4)
 * step in one of several tile shapes, planes per stage x stages in the ring (8x2, 6x2, 4x3, 4x2),
 * all computing every node with the same expressions (the fields agree bit for bit). Autotune times
 * `trial_steps` steps of each from the present state (into the buffer the next step writes, so the
 * state is untouched), keeps the fastest and puts the books and the source's clock back as they
 * were; a grid shape timed once on a device is not timed again in the process. Planes and stages are 0 where the hall does not use that kernel. */
pm_status pm_hall_autotune(pm_hall* h, int trial_steps, int* planes, int* stages);
pm_status pm_hall_set_tile(pm_hall* h, int planes, int stages);
pm_status pm_hall_tile(pm_hall* h, int* planes, int* stages);
pm_status pm_hall_set_stream(pm_hall* h, void* stream);
void pm_hall_destroy(pm_hall* h);

/* ====================================== Room ======================================== */

typedef struct pm_room pm_room;

typedef struct pm_room_desc {
    const char* name;
    double width, height; /* metres */
    int across;           /* nodes along the width (at least 3) */
    double depth;         /* metres: the volume a 2D node stands for */
    double density;       /* kg/m^3 */
    double speed;         /* m/s */
    int precision;        /* pm_precision */
    int device;
} pm_room_desc;

/* Room::new (room.rs:90-120): nx = max(across, 3), dx = width/(nx-1), ny = max(round(height/dx)+1, 3). */
pm_status pm_room_create(const pm_room_desc* desc, pm_room** out);
pm_status pm_room_cells(pm_room* r, int* nx, int* ny, double* dx);
/* Room::released_from (room.rs:140-160) with the profile sampled at the nodes (i + nx j). */
pm_status pm_room_release(pm_room* r, const double* pressure, size_t n);
/* Domain::max_stable_dt (room.rs:361-366): dx/(c sqrt 2), infinite at c = 0. */
pm_status pm_room_max_stable_dt(pm_room* r, double* seconds);
pm_status pm_room_set_tolerance(pm_room* r, double tolerance);
/* `nsteps` calls of Domain::step (room.rs:368-478): the Courant refusal, the half-step start,
 * the startup offset; ledger and audit as for pm_heat_step. */
pm_status pm_room_step(pm_room* r, double dt, long long nsteps, pm_violation* out);
/* total = energy (invariant + startup offset, room.rs:480-482); parts: invariant, offset, datum. */
pm_status pm_room_ledger(pm_room* r, pm_ledger* out);
/* Any pointer may be NULL: p (nx ny), p_prev (nx ny), vx ((nx-1) ny), vy (nx (ny-1)). */
pm_status pm_room_download(pm_room* r, double* p, double* p_prev, double* vx, double* vy);
/* ScalarField::at (room.rs:587-601), the view scene::capture (crates/pantometry-scene/src/lib.rs:
 * 347-420) takes of a room: pressure bilinear between the nodes round each point's (x, y), clamped
 * at the walls, a NaN coordinate reading node 0 along its axis, z not read. Points as for
 * pm_hall_sample. */
pm_status pm_room_sample(pm_room* r, const double lo[3], const double hi[3], const int samples[3], double* out,
                         size_t n);
/* Domain::checkpoint / restore (room.rs:484-505). */
pm_status pm_room_checkpoint(pm_room* r);
pm_status pm_room_restore(pm_room* r);
pm_status pm_room_set_stream(pm_room* r, void* stream);
void pm_room_destroy(pm_room* r);

/* ====================================== Tube ======================================== */

typedef struct pm_tube pm_tube;

typedef struct pm_tube_desc {
    const char* name;
    double length; /* metres */
    int cells;     /* pressure samples along it (at least 3) */
    double area;   /* m^2 */
    double density;
    double speed;
    int precision; /* pm_precision */
    int device;
} pm_tube_desc;

/* Tube::new (lib.rs:167-193): n = max(cells, 3), dx = length/(n-1), both ends closed. */
pm_status pm_tube_create(const pm_tube_desc* desc, pm_tube** out);
pm_status pm_tube_cells(pm_tube* t, int* n, double* dx);
/* Tube::with_ends (lib.rs:211-215, `End` lib.rs:107-116): kind 0 closed, 1 open, 2 matched to
 * the impedance z (z <= 0: the tube's own, rho c). */
pm_status pm_tube_set_ends(pm_tube* t, int left, double z_left, int right, double z_right);
/* Tube::released_from (lib.rs:226-235) with the profile sampled at the n cells. */
pm_status pm_tube_release(pm_tube* t, const double* pressure, size_t n);
/* Domain::max_stable_dt (lib.rs:495-514): dx/c, and dx Z/(2 rho c^2) for an absorbing end. */
pm_status pm_tube_max_stable_dt(pm_tube* t, double* seconds);
/* The per-step audit holds the tube's own books against what its ends published (the
 * `attribute` check of sim.rs:1169-1223): energy plus the published total. */
pm_status pm_tube_set_tolerance(pm_tube* t, double tolerance);
/* `nsteps` calls of Domain::step (lib.rs:516-533, advance lib.rs:386-463). */
pm_status pm_tube_step(pm_tube* t, double dt, long long nsteps, pm_violation* out);
/* total = energy (lib.rs:535-537); parts: energy, published total (`radiated_energy`), datum. */
pm_status pm_tube_ledger(pm_tube* t, pm_ledger* out);
/* Any pointer may be NULL: p (n), p_prev (n), v (n - 1). */
pm_status pm_tube_download(pm_tube* t, double* p, double* p_prev, double* v);
/* Domain::checkpoint / restore (lib.rs:539-554). */
pm_status pm_tube_checkpoint(pm_tube* t);
pm_status pm_tube_restore(pm_tube* t);
pm_status pm_tube_set_stream(pm_tube* t, void* stream);
void pm_tube_destroy(pm_tube* t);

/* ===================================== Bar1D ======================================== */

typedef struct pm_bar pm_bar;

typedef struct pm_bar_desc {
    const char* name;
    int cells;              /* at least 2 */
    double dx;              /* metres per cell */
    double area;            /* cross-section, m^2 */
    pm_substance substance; /* density, conductivity, specific heat, thermal (emissivity unused) */
    double initial_kelvin;  /* every cell, and the temperature the stored heat is measured from */
    int precision;          /* pm_precision */
    int device;
} pm_bar_desc;

/* Bar1D::new (lib.rs:443-464). */
pm_status pm_bar_create(const pm_bar_desc* desc, pm_bar** out);
/* Set / read every cell's temperature (kelvin). An upload re-takes the books from the new state. */
pm_status pm_bar_upload(pm_bar* b, const double* kelvin, size_t n);
pm_status pm_bar_download(pm_bar* b, double* kelvin, size_t n);
/* ScalarField::at (lib.rs:736-751), the view scene::capture takes of a bar: kelvin linear between
 * cell centres along x, the end cell's value beyond either centre and for a NaN x, y and z not
 * read. Points as for pm_hall_sample. */
pm_status pm_bar_sample(pm_bar* b, const double lo[3], const double hi[3], const int samples[3], double* out,
                        size_t n);
/* The heat the next step takes from the bus, handed in by the caller (lib.rs:590-606): lumped
 * joules into the first cell (`take_share` of HEAT), joules per cell (a flux over `exposing`'s
 * faces). Both are booked as taken from the bus. */
pm_status pm_bar_absorb(pm_bar* b, double joules);
pm_status pm_bar_deposit(pm_bar* b, const double* joules, size_t n);
/* Domain::max_stable_dt (lib.rs:564-569): dx^2/(2 alpha). */
pm_status pm_bar_max_stable_dt(pm_bar* b, double* seconds);
/* The per-step audit holds the bar's books (books_balance, lib.rs:555-557): stored heat minus
 * what it took from the bus, the `attribute` check of sim.rs:1169-1223. */
pm_status pm_bar_set_tolerance(pm_bar* b, double tolerance);
/* `nsteps` calls of Domain::step (lib.rs:571-627): the Fourier refusal, the heat handed in (first
 * step only), insulated conduction. */
pm_status pm_bar_step(pm_bar* b, double dt, long long nsteps, pm_violation* out);
/* total = stored heat C sum(T - T_ref) (lib.rs:629-631); parts: stored, absorbed. */
pm_status pm_bar_ledger(pm_bar* b, pm_ledger* out);
/* Domain::checkpoint / restore (lib.rs:633-639): the cells. */
pm_status pm_bar_checkpoint(pm_bar* b);
pm_status pm_bar_restore(pm_bar* b);
pm_status pm_bar_set_stream(pm_bar* b, void* stream);
void pm_bar_destroy(pm_bar* b);

/* ===================================== Cavity ======================================= */

typedef struct pm_cavity pm_cavity;

typedef struct pm_cavity_desc {
    const char* name;
    int nx, ny, nz; /* cells */
    double dx;
    double eps_r, mu_r, sigma; /* the `Medium` (crates/pantometry-em/src/lib.rs:73-118) */
    int precision;             /* pm_precision */
    int device;
} pm_cavity_desc;

/* Cavity::new (cavity.rs:211-245). All walls conducting. */
pm_status pm_cavity_create(const pm_cavity_desc* desc, pm_cavity** out);
/* Cavity::fill once per cell (cavity.rs:250-267): per-cell eps_r, mu_r, sigma (any may be NULL,
 * keeping the present value), then `refresh_media` (cavity.rs:348-458). */
pm_status pm_cavity_fill_cells(pm_cavity* c, const double* eps_r, const double* mu_r,
                               const double* sigma, size_t n);
/* Cavity::obstruct (cavity.rs:281-295): mask[c] != 0 makes cell c a perfect conductor. */
pm_status pm_cavity_obstruct(pm_cavity* c, const uint8_t* mask, size_t n);
/* Cavity::set_boundary (cavity.rs:566-569). wall 0..5 = XLow..ZHigh; kind 0 conducting,
 * 1 magnetic, 2 open (Mur). */
pm_status pm_cavity_set_boundary(pm_cavity* c, int wall, int kind);
/* Cavity::release_mode (cavity.rs:675-732). */
pm_status pm_cavity_release_mode(pm_cavity* c, int m, int p, double amplitude, double dt);
/* Set all six components (host arrays in the reference's index order) and `started`. A new state
 * starts fresh books: nothing dissipated, no source work, the source's clock back at step 0, and
 * the ledger taken from the uploaded fields (the reference has no such setter). */
pm_status pm_cavity_upload(pm_cavity* c, const double* ex, const double* ey, const double* ez,
                           const double* hx, const double* hy, const double* hz, int started);
pm_status pm_cavity_download(pm_cavity* c, double* ex, double* ey, double* ez, double* hx,
                             double* hy, double* hz);
/* Extension (not in the reference): a soft current density current[s] (A/m^2) on the Ez edge
 * with flat index `edge`, applied in step s's electric update; its work is kept in the ledger.
 * An FP32 cavity keeps the six components of a 5^3 box of lattice nodes around the edge in f64
 * (the source's near field, where the pulse moves energy in and out many times over the net work;
 * f32 storage there leaves the books a few 1e-6 of the injected energy off the f64 run), when the
 * box and the edges along its high sides lie a node or more inside the walls, and the cavity is
 * on the padded FP32 layout (one medium, or per-cell epsilon without conductivity or per-cell mu)
 * and not both lossy and obstructed. Elsewhere the FP32 form keeps the whole field in f32. */
pm_status pm_cavity_set_source(pm_cavity* c, long long edge, const double* current, size_t n);
/* Cavity::courant_limit (cavity.rs:1035-1037). */
pm_status pm_cavity_courant_limit(pm_cavity* c, double* seconds);
pm_status pm_cavity_set_tolerance(pm_cavity* c, double tolerance);
/* `nsteps` calls of Domain::step (cavity.rs:1468-1501), ledger and audit per step. */
pm_status pm_cavity_step(pm_cavity* c, double dt, long long nsteps, pm_violation* out);
/* Domain::ledger (cavity.rs:1520-1524). */
pm_status pm_cavity_ledger(pm_cavity* c, pm_ledger* out);
/* Cavity::electric_energy / magnetic_energy (cavity.rs:824-847, 919-940), on the device. */
pm_status pm_cavity_energies(pm_cavity* c, double* electric, double* magnetic);
/* Cavity as a field (cavity.rs:191-206, 735-742): |E| in V/m of the edges of the cell a point falls
 * in, nearest cell, clamped.
 * scene::capture's sampling (crates/pantometry-scene/src/lib.rs:347-420), run on the device over the
 * resident field: `samples[0] * samples[1] * samples[2]` points from `lo` to `hi` (metres, the
 * domain's own coordinates), x fastest, i / (n - 1) of the way along an axis of n > 1 samples and
 * the middle of an axis of one; `out` (host, n values) receives `ScalarField::at` at each point. */
pm_status pm_cavity_sample(pm_cavity* c, const double lo[3], const double hi[3], const int samples[3], double* out,
                           size_t n);
/* Domain::checkpoint / restore (cavity.rs:1566-1590): the fields, `started` and `dissipated`. With
 * a source set (the extension) the checkpoint also keeps the source's clock and its work books, so
 * steps retried after a restore drive the same samples of the current; an FP32 cavity keeps the f64
 * values of its source's near field with them. */
pm_status pm_cavity_checkpoint(pm_cavity* c);
pm_status pm_cavity_restore(pm_cavity* c);
/* No counterpart in the reference. FP32 cavities on the TMA-staged kernel step in one of several
 * tile shapes, planes per stage x stages (one medium: 3x2, 4x2, 3x3; per-cell epsilon: 4x2, 3x2),
 * all computing every edge and face with the same expressions (the fields agree bit for bit).
 * Autotune times `trial_steps` steps of each from the present state (into the buffer the next step
 * writes), keeps the fastest and puts the books and the source's clock back; a grid shape timed once
 * on a device is not timed again in the process. Planes and stages are 0 where the cavity does not
 * use that kernel. A change of media (pm_cavity_fill_cells) goes back to the new form's shape 0. */
pm_status pm_cavity_autotune(pm_cavity* c, int trial_steps, int* planes, int* stages);
pm_status pm_cavity_set_tile(pm_cavity* c, int planes, int stages);
pm_status pm_cavity_tile(pm_cavity* c, int* planes, int* stages);
/* No counterpart in the reference. On the TMA-staged FP32 kernel, when nx is a multiple of 32 and
 * ny of 8, the tiles cover the first nx columns and ny rows of the node lattice and a wall pass in
 * the same launch steps the last column (x = nx) and row (y = ny), whose edges are all wall edges:
 * no tile then runs for one column or row alone. The fields are the same bit for bit either way.
 * On by default; set_wall_split(c, 0) makes the tiles cover the whole lattice. wall_split reports
 * whether the present cavity steps split (0 where it does not use that kernel or does not split). */
pm_status pm_cavity_set_wall_split(pm_cavity* c, int on);
pm_status pm_cavity_wall_split(pm_cavity* c, int* on);
pm_status pm_cavity_set_stream(pm_cavity* c, void* stream);
void pm_cavity_destroy(pm_cavity* c);

/* ============================= Solid3D ensembles (batched) ========================== */

/* Many independent one-material `Solid3D` blocks of uneven sizes, each with its own substance,
 * step and films, advanced together: one persistent kernel per step walks a list of bricks of
 * every block, and runs of 64 steps replay a CUDA graph. It replaces `Ensemble::run` over
 * `Solid3D` samples (crates/pantometry-core/src/ensemble.rs:102-140), each sample driven by
 * `Solid3D::step` (crates/pantometry-thermal/src/solid.rs:1717-1901) with its own ledger
 * (solid.rs:1904-1927). Cells are concatenated block by block, each block in the reference's
 * order i + nx*(j + ny*k). PM_PLAIN_F64 gives each block the bit-exact `Solid3D::step`;
 * PM_FIELDS_F32 stores T - T0 in f32 with FP64 books. */
typedef struct pm_ensemble pm_ensemble;

typedef struct pm_ensemble_grid {
    int nx, ny, nz;
    double dx;
    pm_substance substance;        /* the block's one material (solid.rs:377-421) */
    double initial_kelvin;         /* T0: the start, the ledger's reference and the films' ambient */
    double convection_w_per_m2_k;  /* film on each of the six faces over its whole area
                                      (`losing_from`, solid.rs:1269-1288); 0 = insulated,
                                      +inf = held at T0 (Dirichlet). Emissivity must be 0 with films. */
    double dt;                     /* the block's own step */
} pm_ensemble_grid;

/* `max_stable_dt` of each described block (solid.rs:1709-1715), without a device. */
pm_status pm_ensemble_max_stable_dt(const pm_ensemble_grid* grids, int count, double* seconds);
/* Every block starts at its T0; the brick shape starts at 32 x 8 x 16. */
pm_status pm_ensemble_create(const pm_ensemble_grid* grids, int count, int precision, int device,
                             pm_ensemble** out);
/* kelvin: every block's cells, concatenated in block order. Upload starts fresh books. */
pm_status pm_ensemble_upload(pm_ensemble* e, const double* kelvin, size_t n);
pm_status pm_ensemble_download(pm_ensemble* e, double* kelvin, size_t n);
pm_status pm_ensemble_set_tolerance(pm_ensemble* e, double tol);
/* nsteps steps of every block. Refused before anything moves if a block's dt is past its
 * limit (PM_VIOLATION, "Fourier number"). With a tolerance set, a block whose audit fails stops
 * where it failed (the others go on) and the call returns PM_VIOLATION for the lowest such
 * block, its `site` naming it. */
pm_status pm_ensemble_step(pm_ensemble* e, long long nsteps, pm_violation* out);
/* One pm_ledger per block, in block order (parts: stored, lost, -supplied). */
pm_status pm_ensemble_ledgers(pm_ensemble* e, pm_ledger* out, int count);
/* Brick shape with one cell per thread: x extent 16, 32 or 64 (y = 256 / x) and 8, 16, 32 or 64
 * planes. */
pm_status pm_ensemble_set_shape(pm_ensemble* e, int brick_x, int planes);
/* Any brick shape by its extents in cells: the one-cell shapes above; (f32 only) the shapes whose
 * threads take four adjacent cells of a row each, 16 × 64, 32 × 32, 64 × 16 or 128 × 8; or (plain
 * f64 only) two cells each, 16 × 32, 32 × 16 or 64 × 8; these with 32 or 64 planes. The fields
 * agree bit for bit under every shape. */
pm_status pm_ensemble_set_brick(pm_ensemble* e, int brick_x, int brick_y, int planes);
pm_status pm_ensemble_shape(pm_ensemble* e, int* brick_x, int* brick_y, int* planes);
/* Time `trial_steps` steps of every brick shape on the present state, keep the fastest, and put
 * the state and books back as they were (pm_ensemble_shape gives the chosen y extent). */
pm_status pm_ensemble_autotune(pm_ensemble* e, int trial_steps, int* brick_x, int* planes);
pm_status pm_ensemble_set_stream(pm_ensemble* e, void* stream);
void pm_ensemble_destroy(pm_ensemble* e);

/* ============================ Without allocation ==================================== */

/* No counterpart in the reference. One Hall step (f32 fields, f64 invariant) on device buffers the
 * caller owns, for callers that cannot allocate device memory themselves or through this library —
 * a host that owns every device allocation through its own pool and forbids other allocators, a
 * plugin running inside such a host, or code that must not trigger the device-wide
 * synchronisation cudaMalloc and cudaFree can cause. The kernel is pm_hall_step's; its scratch (a
 * state block and one FP64 partial sum per block) lives in a fixed 64 KiB device array of this
 * library, which every GPU that loads the library holds until the process exits. Grids whose
 * scratch would exceed it are refused with PM_BAD_ARG and a message. Nothing is allocated: no
 * cudaMalloc, no cudaFree, no allocating library call.
 *   Fields are in the reference's index order, nx*ny*nz nodes and (nx-1)*ny*nz, nx*(ny-1)*nz,
 *   nx*ny*(nz-1) faces, as `Hall` lays them out (hall.rs:67-77); the old state is read from
 *   p0/vx0/vy0/vz0 and the new one written to p1/vx1/vy1/vz1; an output that is also an input or
 *   another output is refused with PM_BAD_ARG. first_step != 0 gives the velocities the half step
 *   the leapfrog opens with (hall.rs:427-430). dt must be positive: pm_hall_step, like
 *   `Hall::step` (hall.rs:421-423), treats a non-positive dt as a step that changes nothing, but
 *   this entry point has no state of its own to leave unchanged and returns PM_BAD_ARG. *invariant
 *   receives `invariant_si` of the new state (hall.rs:334-384); the startup offset and the audit
 *   stay with the caller.
 *   The first call on a device looks up the scratch array's device address (cudaGetSymbolAddress,
 *   with that device current); make that first call before any stream capture. Every call shares
 *   the array and leaves its contents behind; each call clears what must start at zero. Calls that
 *   overlap on the GPU (other streams, other threads) race on the array: do not overlap them. */
pm_status pm_hall_step_f32_noalloc(int nx, int ny, int nz, double dx, double speed, double density, double dt,
                                   int first_step, const float* p0, const float* vx0, const float* vy0,
                                   const float* vz0, float* p1, float* vx1, float* vy1, float* vz1, void* stream,
                                   double* invariant);

#ifdef __cplusplus
}
#endif

#endif /* PANTOMETRY_GPU_H */
