/*
 * ldg_b200.h -- C ABI of the B200 Landau-de Gennes Q-tensor solver library (libldg_b200.so).
 *
 * The reference (Spectre71/LCDrSimulator) has no library API: its programs QSR_cuda and
 * KZM_bulk_ldg_cuda launch their kernels directly from main(). Each entry point below
 * replaces one block of that main() and cites it. All entry points:
 *   - take plain pointers and sizes (no C++ or torch types);
 *   - return int status (LDG_OK = 0, LDG_ERR_* otherwise) and never exit or prompt;
 *   - record a message for ldg_last_error() (thread-local) on failure;
 *   - enqueue work on one CUDA stream owned by the handle. qsr_step/kzm_step return after
 *     enqueueing; observe/download/nematic synchronise the stream before returning.
 * A handle must be used from one host thread at a time.
 *
 * Host field layout at the boundary is the reference's: AoS FP64, 5 doubles per cell
 * (Qxx, Qxy, Qxz, Qyy, Qyz), QSR.cuh:22 / KZM_bulk_ldg.cuh:9. Cell order is
 * k + Nz*(j + Ny*i) for the confined solver (QSR.cu:286) and x + Nx*(y + Ny*z) for the
 * periodic bulk solver (KZM_bulk_ldg.cu:161-169). On the device the field is FP32 SoA.
 */
#ifndef LDG_B200_H
#define LDG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define LDG_OK 0
#define LDG_ERR_ARG 1        /* invalid argument or size                        */
#define LDG_ERR_CUDA 2       /* CUDA runtime error (message has the CUDA string) */
#define LDG_ERR_NONFINITE 3  /* a reduction saw a non-finite field value        */
#define LDG_ERR_TIMEOUT 4    /* a bounded device wait gave up                    */
#define LDG_ERR_STATE 5      /* call out of order (e.g. step before upload)      */
#define LDG_ERR_NOMEM 6      /* device allocation failed                         */

/* ------------------------------------------------------------------------------------
 * Confined droplet solver (QSR_cuda)
 * ------------------------------------------------------------------------------------ */
typedef struct qsr_params {
    int Nx, Ny, Nz;                 /* grid, each >= 3 (QSR.cu:1966-1968)                     */
    double dx, dy, dz;              /* spacing in m (QSR.cu:1969-1971)                        */
    double a, b, c, T_star;         /* LdG constants (QSR.cu:1974-1978)                       */
    int bulk_modechoice;            /* 1 = std, 2 = ravnik (QSR.cu:1979, 385-397)             */
    double kappa;                   /* one-constant elastic, used when L1 = L2 = L3 = 0       */
    double L1, L2, L3;              /* anisotropic elastic constants (QSR.cu:2057-2060)       */
    double W;                       /* anchoring: 0 strong, > 0 Rapini-Papoular (QSR.cu:2113) */
    double gamma;                   /* rotational viscosity (QSR.cu:2114)                     */
    double droplet_radius_cells;    /* <= 0: reference radius 0.5*(min(N)-1) (QSR.cu:151)     */
    int compensated;                /* 1: compensated storage (hi + lo FP32 words per value) for
                                       explicit steps: ~48-bit field accumulation, FP32 stencil;
                                       IMEX steps and the direct kernel reset lo to 0           */
} qsr_params;

typedef struct qsr_geometry_info {
    double center_x, center_y, center_z;
    double radius_x, radius_y, radius_z;
    double min_spacing, shell_half_thickness;
    double delta_eff;               /* shell volume / ellipsoid area (QSR.cu:174-185)         */
    long long shell_cells;          /* cells with |sd| <= shell_half_thickness                */
    long long evolving_cells;       /* cells the update touches                               */
    long long active_cells;         /* cells in tiles the step kernel visits (read per step)  */
    long long written_cells;        /* cells the step writes (moving + strongly anchored)     */
    long long box_cells;            /* Nx*Ny*Nz                                               */
} qsr_geometry_info;

typedef struct qsr_step_args {
    double T;                       /* temperature of this step (QSR.cu:2709)                 */
    double S_shell;                 /* shell order of this step (QSR.cu:2711, 1475-1487)      */
    double dt;                      /* time step (QSR.cu:2575-2576)                           */
    double q_norm_cap;              /* 0: off; Frobenius cap of the explicit update (2608)    */
    double noise_sigma;             /* 0: off; Langevin amplitude per component per step      */
    unsigned long long seed;        /* Philox key for the noise                               */
    long long step_index;           /* global index of the first step (noise counter)         */
    int semi_implicit;              /* 1: IMEX Helmholtz-Jacobi update (QSR.cu:2721-2749)     */
    double L_stab;                  /* IMEX stabiliser coefficient                            */
    int jacobi_iters;               /* IMEX Jacobi sweeps per step                            */
} qsr_step_args;

typedef struct qsr_observe_args {
    double T, S_shell;              /* state the energy is evaluated at                       */
    int defects_z_slice;            /* slice of the 2-D defect proxy and checker metric       */
    double defects_S_threshold;     /* default 0.1  (QSR.cu:2634-2644)                        */
    double defects_charge_cutoff;   /* default 0.25                                           */
    int xi_z_slice;                 /* slice of the xi-gradient proxy                         */
    double xi_S_threshold;
    int want_defects;               /* 0 skips the 2-D defect proxy                           */
    int want_xi;                    /* 0 skips the xi proxy                                   */
} qsr_observe_args;

typedef struct qsr_observables {
    double bulk, elastic, anchoring, total;          /* J (QSR.cu:869-992, 654-695)           */
    double radiality; long long radiality_count;     /* QSR.cu:994-1015                       */
    double avg_S, max_S; long long core_count;       /* QSR.cu:2285-2321                      */
    double checker_rel;                              /* NaN unless max_S >= 0.5 (2839-2873)   */
    double defect_density;                           /* NaN when no plaquette (2343-2364)     */
    long long defect_count, defect_plaquettes;
    double xi_grad_proxy; long long xi_edges;        /* QSR.cu:2372-2410                      */
    double max_q_norm;                               /* max Frobenius norm |Q| (debug_dynamics) */
    long long nonfinite_cells;                       /* cells with a non-finite component     */
} qsr_observables;

typedef struct qsr_handle qsr_handle;

/* Replaces the setup block QSR.cu:2141-2226: geometry in FP64, shell mask, delta_eff,
 * device allocations. */
int qsr_create(const qsr_params* params, qsr_handle** out);
int qsr_geometry(const qsr_handle* h, qsr_geometry_info* out);
/* Replaces initializeQTensor / initializeIsotropicWithNoise (QSR.cu:1834-1904): writes the
 * reference's seeded initial field into q_aos5 (host). init_mode 0 random directors, 1 radial,
 * 2 isotropic + N(0, noise_amplitude); std::mt19937(random_seed), random_device if seed < 0. */
int qsr_initial_field(const qsr_handle* h, int init_mode, long long random_seed, double S0,
                      double noise_amplitude, double* q_aos5);
/* Replaces cudaMemcpy H2D of the initial field (QSR.cu:2515, 3078, 3185). */
int qsr_upload(qsr_handle* h, const double* q_aos5);
/* Replaces the D2H of the final / snapshot field (QSR.cu:2930, 2974, 3469). */
int qsr_download(qsr_handle* h, double* q_aos5);
/* Replaces n_steps iterations of the per-step kernel chain: Laplacian, divergence,
 * chemical potential, L3, weak anchoring, update or IMEX, boundary conditions
 * (QSR.cu:2713-2753, 3079-3088, 3234-3249). */
int qsr_step(qsr_handle* h, int n_steps, const qsr_step_args* args);
/* Replaces the log-point observables: reduce_energy (QSR.cu:2323-2341), radiality
 * (2788-2802), nematic avg/max S and checker (2285-2321, 2827-2874), defect proxy
 * (2343-2364) and xi proxy (2372-2410). FP64 reductions, deterministic. */
int qsr_observe(qsr_handle* h, const qsr_observe_args* args, qsr_observables* out);
/* Replaces computeNematicFieldKernel + D2H (QSR.cu:1017-1025, 2816-2821): 4 doubles per
 * cell (S, nx, ny, nz) in the host cell order. */
int qsr_nematic(qsr_handle* h, double* s_n4);
/* Tile autotuner: times each candidate work-item length (planes per tile item) for trial_steps
 * steps with the given step arguments on the uploaded field and keeps the fastest; the field and
 * the launch count are restored afterwards. No counterpart in the reference (fixed launch shapes). */
int qsr_autotune(qsr_handle* h, const qsr_step_args* args, int trial_steps, int* chosen_chunk);
int qsr_sync(qsr_handle* h);
/* The handle's CUDA stream (a cudaStream_t), for timing with events. */
void* qsr_stream(qsr_handle* h);
/* Kernels launched by this handle since creation (launch counter). */
long long qsr_launch_count(const qsr_handle* h);
int qsr_destroy(qsr_handle* h);

/* ------------------------------------------------------------------------------------
 * Ensemble of independent droplets (Kibble-Zurek statistics)
 *
 * Replaces the reference's process-level batching: its tools launch one QSR_cuda process per
 * configuration, one after another (tools/quench_rate_sweep.py:530-537, 664-677). Here all
 * instances advance together: every step is one persistent, work-stealing kernel launch over
 * the active tiles of all instances; K steps are captured once as a CUDA graph and replayed.
 * The step index lives on the device, so each instance's temperature protocol (QSR.cu:
 * 2679-2687), shell order and Philox noise counter are evaluated in the kernel.
 * ------------------------------------------------------------------------------------ */
typedef struct ens_params {
    double dx, dy, dz;
    double a, b, c, T_star;
    int bulk_modechoice;
    double kappa, L1, L2, L3, W, gamma;
    double dt, q_norm_cap;
    int boundary_custom;            /* 1: S_shell = boundary_S, 0: S_eq(T) of each step       */
    double boundary_S;
    int protocol;                   /* 1 step quench, 2 linear ramp (QSR.cu:2437-2447)         */
} ens_params;

typedef struct ens_instance {
    int N;                          /* grid extent along x (and y, z unless set below)         */
    double droplet_radius_cells;
    double T_high, T_low;
    long long pre_equil_iters, ramp_iters;
    unsigned long long seed;        /* Philox key of the instance's noise                      */
    double noise_sigma;             /* per-component Langevin amplitude (0 = off)              */
    int own_material;               /* 1: W, L2, L3 below replace the shared ens_params values */
    double W, L2, L3;
    int Ny, Nz;                     /* grid extents along y and z; 0 = N (cubic)               */
} ens_instance;

typedef struct ens_handle ens_handle;

int ens_create(const ens_params* params, int n_instances, const ens_instance* instances, ens_handle** out);
/* Reference initialisation per instance (QSR.cu:1834-1904) with random_seed = instance seed. */
int ens_initial_fields(ens_handle* h, int init_mode, double S0, double noise_amplitude);
int ens_upload(ens_handle* h, int instance, const double* q_aos5);
int ens_download(ens_handle* h, int instance, double* q_aos5);
/* (S, nx, ny, nz) per cell of one instance, FP64, reference cell order (as qsr_nematic). */
int ens_nematic(ens_handle* h, int instance, double* s_n);
/* Advances every instance by n_steps (replays a captured CUDA graph of n_steps launches). */
int ens_step(ens_handle* h, int n_steps);
/* Observables of one instance at the current step; args NULL: T and S_shell from the
 * instance's protocol, slices Nz/2, thresholds 0.1 / 0.25. */
int ens_observe(ens_handle* h, int instance, const qsr_observe_args* args, qsr_observables* out);
/* Observables of every instance (out[n_instances]) at the current step in one pass: all
 * reductions are enqueued on the ensemble's stream and synchronised once. args: NULL for each
 * instance's defaults (as ens_observe with NULL), else one qsr_observe_args per instance. */
int ens_observe_all(ens_handle* h, const qsr_observe_args* args, qsr_observables* out);
long long ens_step_index(const ens_handle* h);
int ens_geometry(const ens_handle* h, int instance, qsr_geometry_info* out);
/* Times each candidate work-item length (planes per tile item) for trial_steps steps and keeps
 * the fastest; the fields and the step index are restored afterwards. */
int ens_autotune(ens_handle* h, int trial_steps, int* chosen_chunk);
long long ens_cells(const ens_handle* h);           /* total box cells of all instances    */
long long ens_active_cells(const ens_handle* h);    /* cells in visited tiles, all instances */
long long ens_written_cells(const ens_handle* h);
void* ens_stream(ens_handle* h);
long long ens_launch_count(const ens_handle* h);
int ens_destroy(ens_handle* h);

/* ------------------------------------------------------------------------------------
 * Warm-start surrogate: BF16 tcgen05 implicit-GEMM 3x3x3 convolutions (stride 1, zero
 * padding 1). No counterpart in the reference, which has no learned component; these are the
 * layers of the 3-D U-Net that predicts a warm-start Q field for the relaxation.
 * All pointers are DEVICE pointers; work is enqueued on `stream` (NULL = legacy stream).
 * Activations: NDHWC BF16. Weights: [Co][27][Ci] BF16, tap t = 9(dz+1) + 3(dy+1) + (dx+1).
 * Ci in {16, 32, 64, 128, 256}; Co a multiple of 16 in [16, 256].
 * ------------------------------------------------------------------------------------ */
typedef struct sg_conv_shape {
    int N, D, H, W, Ci, Co;
} sg_conv_shape;

/* y = act(conv(x, w) + bias); act 0 = identity, 1 = leaky ReLU (slope 0.01); bias FP32 [Co]
 * or NULL; y BF16, or FP32 when y_fp32 != 0. */
int sg_conv3d_fwd(const sg_conv_shape* s, const void* x, const void* w, const float* bias, void* y, int act,
                  int y_fp32, void* stream);
/* dw[Co][27][Ci] (FP32, overwritten) = sum over voxels of dy (x) shifted x. */
int sg_conv3d_wgrad(const sg_conv_shape* s, const void* x, const void* dy, float* dw, void* stream);
/* wf[Ci][26 - t][Co] = w[Co][t][Ci]: the data gradient of a layer is sg_conv3d_fwd of the
 * output gradient with wf and the shape's Ci and Co exchanged. */
int sg_conv3d_flip_weights(const sg_conv_shape* s, const void* w, void* wf, void* stream);
/* Reads and clears the conv kernels' device error word (LDG_ERR_TIMEOUT when a bounded
 * pipeline wait gave up); synchronises `stream`. */
int sg_check(void* stream);
long long sg_launch_count(void);

/* ------------------------------------------------------------------------------------
 * Periodic bulk solver (KZM_bulk_ldg_cuda)
 * ------------------------------------------------------------------------------------ */
typedef struct kzm_params {
    int Nx, Ny, Nz;                 /* each > 1 (KZM_bulk_ldg.cu:824-826)                     */
    double dx, dy, dz;
    double kappa, gamma;            /* one-constant elastic and viscosity                     */
    double q_norm_cap;              /* 0: off (KZM_bulk_ldg.cu:456-467)                       */
    double defects_S_threshold, defects_charge_cutoff;
} kzm_params;

typedef struct kzm_step_args {
    double A, B, C;                 /* bulk coefficients at this step (KZM_bulk_ldg.cu:919-921) */
    double dt;
    double noise_sigma;             /* sqrt(2/gamma*noise_strength*dt) (KZM_bulk_ldg.cu:955)  */
    unsigned long long seed;
    long long step_index;           /* iteration of the first step (noise counter)           */
} kzm_step_args;

typedef struct kzm_observables {
    double bulk, elastic, total;                     /* per volume (KZM_bulk_ldg.cu:694-696)  */
    double avg_S, max_S;
    double defect_density_per_plaquette, defect_line_density, xi_grad_proxy;
    long long defect_plaquettes_used, nonzero_defect_plaquettes;
} kzm_observables;

typedef struct kzm_handle kzm_handle;

/* Replaces KZM_bulk_ldg.cu:895-899 (allocation and upload of the field). */
int kzm_create(const kzm_params* params, kzm_handle** out);
int kzm_upload(kzm_handle* h, const double* q_aos5);
int kzm_download(kzm_handle* h, double* q_aos5);
/* Replaces n_steps iterations of updateBulkLdgKernel + swap (KZM_bulk_ldg.cu:951-970). */
int kzm_step(kzm_handle* h, int n_steps, const kzm_step_args* args);
/* Replaces the full D2H + host compute_observables (KZM_bulk_ldg.cu:923-925, 543-713). */
int kzm_observe(kzm_handle* h, double A, double B, double C, kzm_observables* out);
/* No counterpart in the reference. The observables of kzm_observe computed straight from a
 * field the caller keeps in device memory (the reference's own layout: AoS FP64, 5 doubles per
 * site, x fastest), for callers that must not allocate device memory: code running inside
 * another framework that has reserved the GPU's memory for its own pool (a cudaMalloc there can
 * fail, or take memory the pool expects to own), and step loops that cannot afford the device
 * synchronisation that cudaMalloc/cudaFree imply. It calls no cudaMalloc/cudaFree: its scratch
 * is a fixed file-scope device array in this library (16 MiB, held on every GPU that loads the
 * library until the process exits), sized for at most KZM_NOALLOC_MAX_SITES sites (larger grids
 * get LDG_ERR_ARG before any device work). The first call on each device looks up that array's
 * device address, so make that first call before any stream capture. All calls share the
 * array: calls that overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. Work runs on `stream` (a cudaStream_t of the current device,
 * NULL = legacy default stream; a stream of another device gets LDG_ERR_ARG); the call
 * synchronises it before returning the observables. */
#define KZM_NOALLOC_MAX_SITES (1LL << 19)
int kzm_observe_device_noalloc(const kzm_params* params, const double* q_aos5_device, double A, double B,
                               double C, void* stream, kzm_observables* out);
void* kzm_stream(kzm_handle* h);
long long kzm_launch_count(const kzm_handle* h);
int kzm_destroy(kzm_handle* h);

/* ------------------------------------------------------------------------------------ */
const char* ldg_last_error(void);
const char* ldg_version(void);

#ifdef __cplusplus
}
#endif
#endif
