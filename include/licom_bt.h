/*
 * licom_bt.h - C-ABI of the B200 barotropic duogrid solver (libbt.so).
 *
 * The reference integrates the barotropic shallow-water equations with
 * `_barotr_rk2_core(state, consts, nbb, dtb, px, py)` /
 * `_barotr_rk3_core(...)` (src/licom/momentum/barotr.py:41-87), compiled once
 * per run by `Schedule.configure` -> `make_spmd_jit`
 * (src/licom/mymodule/schedule.py:209-243, src/licom/kernel/spmd.py:38-75)
 * and called from `schedule_core` (schedule.py:148-190).  This library is the
 * compiled form of that path on one GPU: a plan captures the 17 constants
 * once (like the JIT's closure-captured consts) and every round advances a
 * state by nbb substeps.
 *
 * Conventions
 *   - Every field is a device array (6, M, M), M = N + 6, C order, in the
 *     plan's dtype; matrices are (6, M, M, 2, 2), k2e_coef is (6, M, M, 2),
 *     the k2e location tables are int32 (6, M, M).  Axis -2 is the Fortran i
 *     index, axis -1 the Fortran j index.
 *   - Calls are stream-ordered and non-blocking; pass a cudaStream_t as void*
 *     (NULL = the legacy default stream).
 *   - Every call returns BT_OK (0) or a negative code and never aborts; the
 *     message is available from bt_last_error() (thread-local).
 *   - A plan is not thread-safe: use one plan per host thread / stream.
 */
#ifndef LICOM_BT_H
#define LICOM_BT_H

#ifdef __cplusplus
extern "C" {
#endif

#define BT_OK 0
#define BT_EINVAL -1   /* bad argument (shape, dtype, pointer, option) */
#define BT_ENOMEM -2   /* device or host allocation failed */
#define BT_ECUDA -3    /* a CUDA runtime call failed */
#define BT_EDEVICE -4  /* a kernel reported an error through the plan's device flag */
#define BT_ENOTSUP -5  /* valid input the solver does not support */

#define BT_F64 0
#define BT_F32 1

/* Round execution modes */
#define BT_MODE_STREAM 0      /* kernels launched in stream order */
#define BT_MODE_GRAPH 1       /* the round is captured once as a CUDA graph and replayed */
#define BT_MODE_PERSISTENT 2  /* one cooperative launch with grid barriers per round */
#define BT_MODE_RESIDENT 3    /* one cooperative launch per round, one CTA per tile holding its constants
                                 and face cache on chip, neighbour tiles synchronised by progress flags;
                                 grids whose tiles all fit on the GPU at once (else BT_ENOTSUP) */

/* Plan options (bt_plan_set_option) */
#define BT_OPT_MAX_CTAS 1    /* persistent mode: cap on the cooperative grid (0 = occupancy limit) */
#define BT_OPT_SPIN_LIMIT 2  /* persistent / resident mode: polls a grid-barrier or neighbour wait may
                                take before it gives up */
#define BT_OPT_KERNEL_TIMING 3  /* 1 = bracket the round kernel (persistent / resident mode) or each phase
                                   kernel (stream mode) with CUDA events on its stream; setting it resets
                                   the record */
#define BT_OPT_FULL_TILES 4  /* stream / graph mode, which phase kernels run: -1 (default) by size, the
                                kernels with a path specialised for full interior tiles when a launch
                                takes more than one wave of CTAs and the smaller edge-path-only kernels
                                otherwise; 1 = always the former, 0 = always the latter (same results) */

/* Kernel kinds of bt_plan_kernel_time */
#define BT_KERNEL_ROUND 0     /* the persistent or resident round kernel */
#define BT_KERNEL_PHASE_H 1   /* the h-update tile kernel of a stage */
#define BT_KERNEL_PHASE_UV 2  /* the momentum-update tile kernel of a stage */

/* Plan information (bt_plan_get_info) */
#define BT_INFO_LAST_GRID 1      /* CTAs of the last persistent launch */
#define BT_INFO_SCRATCH_BYTES 2  /* device scratch owned by the plan */
#define BT_INFO_FULL_TILES 3     /* stream / graph mode phase kernels at the plan's tile and size: bit 0 set =
                                    phase H runs the kernel with the full-tile path, bit 1 = phase UV */

typedef struct bt_plan bt_plan;

/* Geometry of one resolution: the 17 constants in CONST_SOURCES order
 * (src/licom/mymodule/schedule.py:95-116), as device pointers. */
typedef struct bt_grid_desc {
  int n;      /* cells per face edge N (>= 4) */
  int dtype;  /* BT_F64 or BT_F32 */
  const void* dzph_x;
  const void* dzph_y;
  const void* rdx;
  const void* rdy;
  const void* a_f;
  const void* k2e_coef;
  const int* loc_i_local;
  const int* loc_j_local;
  const void* a_c2l;
  const void* a_l2c;
  const void* inner;
  const void* outer;
  const void* a_gct;
  const void* a_sina;
  const void* rda;
  const void* c_dy;
  const void* d_dx;
} bt_grid_desc;

/* Round input: STATE_KEYS[0:6] = h0, h0p, ub, vb, ubp, vbp
 * (src/licom/mymodule/schedule.py:62-92).  h0p/ubp/vbp may alias h0/ub/vb. */
typedef struct bt_state_in {
  const void* h0;
  const void* h0p;
  const void* ub;
  const void* vb;
  const void* ubp;
  const void* vbp;
} bt_state_in;

/* Round output.  h0/ub/vb receive the new state (also the new h0p/ubp/vbp,
 * barotr.py:59) with halos filled; they must not alias any input.  diag[0..9]
 * receive STATE_KEYS[6:16] (celerity_x, celerity_y, ub_ct, vb_ct, ub_cx,
 * ub_cy, vb_cx, vb_cy, advx, advy) of the last stage; pass NULL in diag[0]
 * to skip the diagnostics. */
typedef struct bt_state_out {
  void* h0;
  void* ub;
  void* vb;
  void* diag[10];
} bt_state_out;

/* Build a plan: validates the masks, builds the halo gather tables from
 * k2e_coef/loc_i/loc_j and the cube topology, allocates the stage scratch.
 * Replaces Schedule.configure/make_spmd_jit (schedule.py:209-243, spmd.py:38-75)
 * and Communication.configure (src/licom/kernel/communication.py:269-291).
 * The constant arrays must stay alive and unchanged while the plan exists;
 * the 2x2 matrix arrays a_c2l, a_l2c and a_gct must start on a 16-byte
 * boundary (BT_EINVAL otherwise). */
int bt_plan_create(const bt_grid_desc* desc, bt_plan** out);

/* Release a plan and everything it owns (no counterpart: JAX frees by refcount). */
int bt_plan_destroy(bt_plan* plan);

/* Tile shape (rows ti x columns tj of interior cells per CTA) and round mode. */
int bt_plan_set_tile(bt_plan* plan, int ti, int tj);
int bt_plan_set_mode(bt_plan* plan, int mode);

/* Set a plan option (BT_OPT_*).  A barrier wait that exceeds BT_OPT_SPIN_LIMIT
 * polls sets the plan's device error flag and ends the round early instead of
 * waiting forever; bt_check_device_error then reports BT_EDEVICE. */
int bt_plan_set_option(bt_plan* plan, int key, long long value);

/* Sum of the durations of the timed kernels of one kind (BT_KERNEL_*) launched
 * since BT_OPT_KERNEL_TIMING was last set; waits for them. */
int bt_plan_kernel_time(bt_plan* plan, int kind, double* ms_total, int* launches);

/* Read plan information (BT_INFO_*); -1 for an unknown key. */
long long bt_plan_get_info(bt_plan* plan, int key);

/* Advance nbb (>= 1) substeps of RK2 (rk = 2, midpoint, barotr.py:41-61) or
 * RK3 (rk = 3, barotr.py:64-87) with step dtb.  Replaces the call
 * rk_core(barotr_s, barotr_consts, nbb, dtb, px, py) (schedule.py:170) with
 * px = py = 1; STATE_KEYS[16:23] pass through untouched and are not handled here. */
int bt_round(bt_plan* plan, const bt_state_in* in, const bt_state_out* out, int nbb, double dtb,
             int rk, void* stream);

/* One RK stage: _step_rk_logic(h0, h0p, ub, vb, ubp, vbp, consts, dt, beta_d,
 * is_laststep, px, py) (src/licom/momentum/barotr_pure.py:100-168).  The
 * inputs' halo cells are used as given; out->h0/ub/vb receive new_h0/new_ub/
 * new_vb with filled halos, out->diag[0..9] the ten diagnostics of the stage
 * (computed from its inputs), or pass diag[0] = NULL to skip them. */
int bt_stage(bt_plan* plan, const bt_state_in* in, const bt_state_out* out, double dt, double beta_d,
             int is_laststep, void* stream);

/* Fill the halo cells of a scalar field h and/or a vector (u, v) from their
 * interiors: ext_scalar / ext_vector (src/licom/kernel/cube.py:130-153).
 * Any of h, u (with v) may be NULL. */
int bt_fill_halo(bt_plan* plan, void* h, void* u, void* v, void* stream);

/* Edge average of the face-normal C-grid components of (u, v) in place:
 * Communication.boundary_communication (communication.py:504-570). */
int bt_edge_average(bt_plan* plan, void* u, void* v, void* stream);

/* Host-only: the halo gather tables a plan builds, for inspection and testing.
 * For n cells per face edge (M = n + 6, nh = 12 n + 36 halo cells per face):
 * src (6*nh*2 int32, absolute source cell offsets within a (6,M,M) field),
 * weights (6*nh*2), route (24 packed entries nb | side << 4 | rev << 6).
 * Halo cell (i, j) of face f has index f*nh + id, id numbering rows 0..2,
 * rows M-3..M-1 (all columns), then the W and E bands row by row.  Together
 * with the c2l/l2c rotations these tables reproduce ext_scalar/ext_vector
 * (cube.py:40-153) and the halo routing of communication.py:269-474. */
int bt_halo_table_host(int n, const double* k2e_coef, const int* loc_i, const int* loc_j, int* src,
                       double* weights, int* route);

/* Interior statistics of a (6, n+6, n+6) field: out3 (device, 3 float64) =
 * max, min, mean over the 6 n^2 interior cells; the global diagnostic of
 * src/licom/mymodule/diag.py:45-75 computed on the device.  Deterministic. */
int bt_interior_stats(int n, int dtype, const void* field, void* out3, void* stream);

/* Conservation sums over the interior: out2 (device, 2 float64) = total mass
 * sum(h da) and energy sum((g h^2 / 2 + (depth + h) |u_lonlat|^2 / 2) da),
 * da = 1 / rda, u_lonlat = a_c2l . (u, v).  Terms in the fields' precision,
 * sums compensated in float64, fixed reduction order (deterministic).
 * No counterpart in the reference (its diagnostics stop at max/min/mean). */
int bt_conservation(int n, int dtype, const void* h, const void* u, const void* v, const void* rda,
                    const void* a_c2l, double depth, void* out2, void* stream);

/* bt_round without any allocation, for callers that cannot allocate device
 * memory (a runtime's custom-call handler given only its operand buffers, a
 * model driver that reserves its GPU memory up front, a service whose memory
 * footprint is fixed once it serves).  No counterpart in the reference.
 * Same arguments and results as bt_round, but no plan: desc is passed directly
 * and the halo tables are rebuilt on the device each call, stream-ordered.
 * All scratch lives in one 6 MiB array the library declares statically
 * (held by every GPU that loads the library until exit).  Largest sizes:
 * float64 N <= 112 (rk 2) / 96 (rk 3), float32 N <= 160 (rk 2) / 136 (rk 3);
 * larger sizes return BT_EINVAL.  The first call on a device sets up the
 * array's address and must come before any stream capture.  The first call
 * with a given set of constant pointers on a device checks the tables as
 * bt_plan_create does (k2e locations inside the band: BT_EINVAL; inner/outer
 * the exact masks: BT_ENOTSUP) and synchronises the stream to read the
 * result; later calls with the same pointers skip the check, so the tables
 * must not change meanwhile.  Calls share the array: calls whose GPU work
 * overlaps race and must be serialised.  The round runs the 8 x 16 tile shape
 * whatever bt_plan_set_tile a plan would use (float64 results are the same for
 * every shape).  As for bt_plan_create, a_c2l, a_l2c and a_gct must start on a
 * 16-byte boundary (BT_EINVAL otherwise). */
int bt_round_noalloc(const bt_grid_desc* desc, const bt_state_in* in, const bt_state_out* out, int nbb,
                     double dtb, int rk, void* stream);

/* Synchronise the plan's work and report a device-side error flag, if set. */
int bt_check_device_error(bt_plan* plan);

const char* bt_last_error(void);
int bt_version(void);

/* ---- Batched rounds: many independent integrations in one launch ----------
 * No counterpart in the reference, which advances one state per call
 * (rk_core, schedule.py:170); a batch replaces a loop of such calls over
 * ensemble members or served requests.  Members may differ in resolution
 * (one plan per resolution supplies the geometry; several members may share
 * a plan), in dtb and in substep count: a round advances member k by its own
 * nbb substeps, members with fewer substeps retire early and the launch's
 * later phases cover only the members still running.  Each member's result
 * is the one bt_round gives for the same input (same tile shape and dtype). */
typedef struct bt_batch bt_batch;

typedef struct bt_member {
  bt_plan* plan;       /* geometry of the member's resolution; dtype must match the batch */
  bt_state_in in;      /* as bt_round */
  bt_state_out out;    /* as bt_round; diag[0] = NULL skips the diagnostics */
  void* scratch;       /* device buffer of bt_member_scratch_bytes, 256-byte aligned, private to the member */
  int nbb;             /* substeps of this round (>= 1) */
  double dtb;
} bt_member;

/* Device scratch one member needs for RK order rk (stage fields and face caches). */
int bt_member_scratch_bytes(bt_plan* plan, int rk, unsigned long long* bytes);

/* A batch of dtype BT_F64 / BT_F32 taking up to max_members members per call,
 * on the current device.  Default mode BT_MODE_PERSISTENT (one cooperative
 * launch per round: all phases of all members, grid barriers between phases,
 * halo fills and diagnostics at the end); BT_MODE_STREAM launches one kernel
 * per phase over all active members instead.  Tile shape default 8 x 32. */
int bt_batch_create(int dtype, int max_members, bt_batch** out);
int bt_batch_destroy(bt_batch* batch);
int bt_batch_set_mode(bt_batch* batch, int mode);
int bt_batch_set_tile(bt_batch* batch, int ti, int tj);
/* BT_OPT_MAX_CTAS and BT_OPT_SPIN_LIMIT, as for plans. */
int bt_batch_set_option(bt_batch* batch, int key, long long value);
/* BT_INFO_LAST_GRID; -1 for an unknown key. */
long long bt_batch_get_info(bt_batch* batch, int key);

/* Advance every member by its nbb substeps of RK order rk (2 or 3), stream
 * ordered.  The member array is read during the call only.  The host may
 * block when four earlier calls on this batch are still running on the GPU. */
int bt_batch_round(bt_batch* batch, const bt_member* members, int count, int rk, void* stream);

/* Synchronise the device and report the batch's device error flag, if set. */
int bt_batch_check_device_error(bt_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* LICOM_BT_H */
