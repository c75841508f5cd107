/*
 * lddmm_b200.h -- C ABI of the B200-native point-set hot path of py-lddmm.
 *
 * Conventions (every entry point):
 *  - Arrays are float64, C-contiguous, on the CUDA device of `stream` (device pointers), in the reference's
 *    layout: points / momenta / covectors are (N, 3) row-major (numpy `float64 (N,3)`), trajectories are
 *    (T+1, N, 3), faces are int64 (F, 3). Outputs are written, never accumulated into, and never alias inputs.
 *  - One kernel width `sigma` per call (Gaussian, or the Laplacian family where an entry point takes `kernel`),
 *    with the reference's default `ms_exponent = -1` weighting; multi-scale kernels are one call per width.
 *  - `origin` (host pointer to 3 doubles, may be NULL = 0): coordinates are centred on it before the FP32
 *    conversion. Results are translation invariant; pass the centroid of the points for best FP32 accuracy.
 *    The Gaussian FP32 kernels of lddmm_apply_k, the second-order forward step, the surface energies and the
 *    varifold / measure gradients centre every target block on its own in FP64 and do not depend on it.
 *  - `precision`: LDDMM_FP32C = FP32 pair arithmetic with compensated (two-sum) accumulation across tiles and
 *    FP64 epilogues; LDDMM_FP64 = the same kernels in FP64 (the faithful baseline).
 *  - `workspace` / `workspace_bytes`: caller-provided device scratch of at least
 *    lddmm_workspace_bytes(n_max, m_max, precision) bytes. No entry point allocates memory.
 *  - Calls are asynchronous on `stream`, launch no host synchronisation and are safe to capture in a CUDA graph.
 *  - Return value: LDDMM_OK or an error status; argument errors are detected before any launch.
 */
#ifndef LDDMM_B200_H
#define LDDMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* lddmm_stream_t; /* == cudaStream_t */

enum {
  LDDMM_OK = 0,
  LDDMM_ERR_INVALID_ARGUMENT = 1,
  LDDMM_ERR_LAUNCH = 2,
  LDDMM_ERR_NONFINITE = 3, /* reserved: entry points never read results back, so NaN / Inf propagate to the
                               outputs as in the reference */
  LDDMM_ERR_WORKSPACE = 4,
  LDDMM_ERR_CUDA = 5,
  LDDMM_ERR_UNSUPPORTED = 6
};

enum { LDDMM_FP32C = 0, LDDMM_FP64 = 1 };

/* Kernel family (`kernel` argument): the Gaussian exp(-r^2 / (2 sigma^2)) (KernelSpec name 'gauss'), or the
 * reference's 'laplacian' kernel of order q = 0..4, P_q(r / sigma) exp(-r / sigma) with the polynomials lapPol /
 * lapPolDiff / lapPolDiff2 of base/kernelFunctions_util.py:20-56 (KernelSpec(name='laplacian', order=q),
 * base/kernelFunctions.py:363-368). */
enum { LDDMM_KERNEL_GAUSS = 0, LDDMM_KERNEL_LAPLACIAN_0 = 16, LDDMM_KERNEL_LAPLACIAN_4 = 20 };
#define LDDMM_KERNEL_LAPLACIAN(order) (LDDMM_KERNEL_LAPLACIAN_0 + (order))

/* Library version and self description. */
const char* lddmm_version(void);
const char* lddmm_status_string(int status);

/* Scratch size (bytes) sufficient for every entry point with at most n_max targets and m_max sources. */
size_t lddmm_workspace_bytes(int64_t n_max, int64_t m_max, int precision);

/* ---------------------------------------------------------------------------------------------------------
 * Kernel operators (replace Kernel.* in base/kernelFunctions.py:452-674 and the numba / pykeops backends
 * ku.applyK / applyDiffKT / applyDDiffK / applykdiff1and2 / applyDiv / applyktensor in
 * base/kernelFunctions_util.py:443-1506). y: (n,3) targets, x: (m,3) sources. `kernel`: LDDMM_KERNEL_GAUSS or
 * LDDMM_KERNEL_LAPLACIAN(order) (LDDMM_ERR_INVALID_ARGUMENT otherwise).
 * ------------------------------------------------------------------------------------------------------- */

/* out(n,3) = K(y, x) a.  Kernel.applyK(x, a, firstVar=y)  base/kernelFunctions.py:452.
 * When y == x (the same pointer) and n == m, FP32 evaluates the self-sum once per unordered pair (symmetric
 * kernel; the workspace of lddmm_workspace_bytes(n, n, ...) covers it); results agree with the ordered-pair
 * evaluation to FP32 rounding. */
int lddmm_apply_k(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma, int kernel,
                  const double* origin, double* out, int precision, void* workspace, size_t workspace_bytes,
                  lddmm_stream_t stream);

/* out(n,3) = DK^T.  Kernel.applyDiffKT(x, p, a, firstVar=y, regweight, lddmm, sym)  base/kernelFunctions.py:581.
 * mode 0 = plain (p: (n,3), a: (m,3)); 1 = sym; 2 = lddmm (sym / lddmm need n == m, p and a both (n,3)). */
int lddmm_apply_diff_kt(const double* y, int64_t n, const double* x, const double* p, const double* a, int64_t m,
                        double sigma, int kernel, int mode, double regweight, const double* origin, double* out,
                        int precision, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* out(n,3) = DDK_{11 and 12}(x; nn, a, p).  Kernel.applyDDiffK11and12(x, n, a, p)  base/kernelFunctions.py:665. */
int lddmm_apply_ddiff_k11and12(const double* x, const double* nn, const double* a, const double* p, int64_t n,
                               double sigma, int kernel, const double* origin, double* out, int precision,
                               void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* out(n,3) = DK_{1 and 2}(x; a1, a2).  Kernel.applyDiffK1and2(x, a1, a2)  base/kernelFunctions.py:549. */
int lddmm_apply_diff_k1and2(const double* x, const double* a1, const double* a2, int64_t n, double sigma, int kernel,
                            const double* origin, double* out, int precision, void* workspace, size_t workspace_bytes,
                            lddmm_stream_t stream);

/* out(n) = divergence of K(., x) a at y.  Kernel.applyDivergence(x, a, firstVar=y)  base/kernelFunctions.py:638. */
int lddmm_apply_divergence(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma,
                           int kernel, const double* origin, double* out, int precision, void* workspace,
                           size_t workspace_bytes, lddmm_stream_t stream);

/* out(n) = sum_l K(y_k, x_l) (ay_k ax_l + (by_k.bx_l)^2) with the Gaussian K.  Kernel.applyKTensor
 * base/kernelFunctions.py:509. */
int lddmm_apply_k_tensor(const double* y, int64_t n, const double* x, int64_t m, const double* ay, const double* ax,
                         const double* by, const double* bx, double sigma, const double* origin, double* out,
                         int precision, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* out(n,3) = K(y, x) a without any workspace argument and without allocating: lddmm_apply_k for callers that
 * cannot allocate device memory at call time (an application whose device-memory budget is fixed at start-up, a
 * plugin host that gives its plugins no allocator, or a latency-critical path that may not call cudaMalloc because
 * it can synchronise the device). This entry point has no counterpart in the reference.
 * Its scratch is a 32 MiB array built into the library; every GPU that loads the library holds it until exit.
 * Limits: n <= 262,144 targets. The scratch is the sum's partial slots only and does not grow with the number of
 * sources: on a B200 every request with at most 262,144 targets fits (20.7 MiB at most) for any source count up to
 * the library's limit of 536,870,911. A request whose scratch would not fit the array (a device with many more
 * resident CTAs) is rejected with LDDMM_ERR_WORKSPACE before any launch. The first call on a device looks up the
 * array's address with that device current: make it before any stream capture. All calls share the array (nothing needs clearing between calls);
 * calls that overlap on the GPU race on it and must be serialised by the caller. */
int lddmm_apply_k_static(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma,
                         const double* origin, double* out, int precision, lddmm_stream_t stream);

/* Dense-weight variants (O(n m) weights streamed from HBM).
 * out(n,d) = sum_l K(y_k, x_l) u[k,l,:]  -- Kernel.applyK(matrixWeights=True) -> ku.applykmat  kernelFunctions_util.py:1509
 * out(n,3) = sum_l -(y_k-x_l)/sigma^2 K beta[k,l] -- Kernel.applyDiffKmat -> ku.applykdiffmat  kernelFunctions_util.py:1631 */
int lddmm_apply_k_mat(const double* y, int64_t n, const double* x, int64_t m, const double* u, int64_t d, double sigma,
                      double* out, lddmm_stream_t stream);
int lddmm_apply_diff_k_mat(const double* y, int64_t n, const double* x, int64_t m, const double* beta, double sigma,
                           double* out, lddmm_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Landmark shooting and adjoint (replace base/pointEvolution.py). Fused kernels share one exp per pair.
 * `kernel`: LDDMM_KERNEL_GAUSS or LDDMM_KERNEL_LAPLACIAN(order), as for the kernel operators.
 * ------------------------------------------------------------------------------------------------------- */

/* One second-order (geodesic) Euler step: x1 = x + dt K(x)a, a1 = a - dt DK^T(x; a, a).
 * secondOrderEvolution loop body, base/pointEvolution.py:433-449. */
int lddmm_second_order_step(const double* x, const double* a, int64_t n, double sigma, int kernel, double dt,
                            const double* origin, double* x_next, double* a_next, int precision, void* workspace,
                            size_t workspace_bytes, lddmm_stream_t stream);

/* Second-order shooting over T steps of size dt: xt, at (T+1,n,3) with xt[0]=x0, at[0]=a0.
 * secondOrderEvolution  base/pointEvolution.py:385. */
int lddmm_second_order_shoot(const double* x0, const double* a0, int64_t n, int64_t T, double sigma, int kernel,
                             double dt, const double* origin, double* xt, double* at, int precision, void* workspace,
                             size_t workspace_bytes, lddmm_stream_t stream);

/* One adjoint step (base/pointEvolution.py:539-546):
 * px_prev = px + dt [DK^T_sym(x; px, a) - DDK11and12(x; a, a, pa)],  pa_prev = pa + dt [K(x) px - DK1and2(x; pa, a)]. */
int lddmm_second_order_adjoint_step(const double* x, const double* a, const double* px, const double* pa, int64_t n,
                                    double sigma, int kernel, double dt, const double* origin, double* px_prev,
                                    double* pa_prev, int precision, void* workspace, size_t workspace_bytes,
                                    lddmm_stream_t stream);

/* Row-range forms for sharding one time step over several GPUs (targets = rows row0 .. row0+nrows-1 of the full
 * state, sources = all n rows; outputs are the nrows new rows). Same sums as the whole-step entry points above
 * (base/pointEvolution.py:433-449 and :539-546); workspace: lddmm_workspace_bytes(nrows, n, precision). */
int lddmm_second_order_step_rows(const double* x, const double* a, int64_t n, int64_t row0, int64_t nrows, double sigma,
                                 int kernel, double dt, const double* origin, double* x_next_rows, double* a_next_rows,
                                 int precision, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);
int lddmm_second_order_adjoint_step_rows(const double* x, const double* a, const double* px, const double* pa,
                                         int64_t n, int64_t row0, int64_t nrows, double sigma, int kernel, double dt,
                                         const double* origin, double* px_prev_rows, double* pa_prev_rows,
                                         int precision, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* Full adjoint sweep + gradient: given xt, at (T+1,n,3) and px1, pa1 (n,3), writes pxt, pat (T+1,n,3) and
 * da0 = K(x0) a0 - pat[0].  secondOrderCovector / secondOrderGradient  base/pointEvolution.py:489-618. */
int lddmm_second_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                                double dt, const double* px1, const double* pa1, const double* origin, double* pxt,
                                double* pat, double* da0, int precision, void* workspace, size_t workspace_bytes,
                                lddmm_stream_t stream);

/* First-order shooting x_{t+1} = x_t + dt K(x_t) a_t with dt = 1/T, and the kinetic energy
 * energy[0] = regweight * dt * sum_t a_t . K(x_t) a_t (device scalar, FP64, deterministic order).
 * landmarkDirectEvolutionEuler base/pointEvolution.py:88 + SurfaceMatching.objectiveFunDef base/surfaceMatching.py:546.
 * `energy` may be NULL. */
int lddmm_first_order_shoot(const double* x0, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                            double regweight, const double* origin, double* xt, double* energy, int precision,
                            void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* First-order adjoint + gradient (landmarkHamiltonianCovector/Gradient base/pointEvolution.py:167-236 and the
 * in-class copy base/surfaceMatching.py:728-908): p_t = p_{t+1} + dt DK^T_lddmm(x_t; p_{t+1}, a_t), and
 *   dat_t = 2 regweight a_t - p_{t+1}            (euclidean = 0)
 *   dat_t = K(x_t)(2 regweight a_t - p_{t+1})    (euclidean = 1, the BFGS gradient of SurfaceMatching).
 * Both sums of a step share one exp per pair. pxt (T+1,n,3), dat (T,n,3). */
int lddmm_first_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma, int kernel,
                               double regweight, const double* px1, int euclidean, const double* origin, double* pxt,
                               double* dat, int precision, void* workspace, size_t workspace_bytes,
                               lddmm_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Surface data terms (replace base/surfaceDistances.py). `weights` are per-vertex weights (may be NULL = 1);
 * face weights are their face means (base/surfaces.py:326-351).
 * kind: LDDMM_DATA_VARIFOLD (unoriented, f0 = 1 + u^2), LDDMM_DATA_CURRENT, LDDMM_DATA_MEASURE.
 * ------------------------------------------------------------------------------------------------------- */
enum { LDDMM_DATA_VARIFOLD = 0, LDDMM_DATA_CURRENT = 1, LDDMM_DATA_MEASURE = 2 };

/* Scratch size (bytes) for lddmm_surface_energy / lddmm_surface_gradient with nf deformed and nf1 target faces. */
size_t lddmm_surface_workspace_bytes(int64_t nf, int64_t nf1, int precision);

/* energy[0] = |def|^2 - 2 <def, tgt>  (xNormDef), energy[1] = |tgt|^2 (xNorm0); device scalars, FP64.
 * varifoldNormDef / varifoldNorm0  base/surfaceDistances.py:286-382 (current :22-81, measure :207-223). */
int lddmm_surface_energy(int kind, const double* xdef, int64_t nv, const int64_t* faces, int64_t nf,
                         const double* weights, const double* x1, int64_t nv1, const int64_t* faces1, int64_t nf1,
                         const double* weights1, double sigma, const double* origin, int with_norm0, double* energy,
                         int precision, void* workspace, size_t workspace_bytes, lddmm_stream_t stream);

/* Vertex gradient of xNormDef: px (nv,3) and, for the varifold when pxw != NULL, the vertex-weight gradient
 * pxw (nv) (varifoldNormGradient(with_weights=True)). The faces->vertices scatter is a deterministic gather
 * through the vertex->(face, corner) table `vf_offsets` (nv+1, int32) / `vf_items` (3*nf, int32, item =
 * 3*face + corner), built once per topology by lddmm_vertex_face_table.
 * varifoldNormGradient base/surfaceDistances.py:394-573 (current :90-133, measure :232-278). */
int lddmm_surface_gradient(int kind, const double* xdef, int64_t nv, const int64_t* faces, int64_t nf,
                           const double* weights, const int32_t* vf_offsets, const int32_t* vf_items, const double* x1,
                           int64_t nv1, const int64_t* faces1, int64_t nf1, const double* weights1, double sigma,
                           const double* origin, double* px, double* pxw, int precision, void* workspace,
                           size_t workspace_bytes, lddmm_stream_t stream);

/* Host-side helper (HOST pointers): vertex -> (face, corner) incidence table in ascending (face, corner) order. */
int lddmm_vertex_face_table(const int64_t* faces_host, int64_t nf, int64_t nv, int32_t* vf_offsets_host,
                            int32_t* vf_items_host);

/* ---------------------------------------------------------------------------------------------------------
 * Learned momentum proposal (no counterpart in the reference, which has no learned component). Per-vertex MLP
 * with BF16 weights / activations and FP32 accumulation on the tensor cores.
 * ------------------------------------------------------------------------------------------------------- */

/* C = epilogue(op(A) op(B)): A is (M,K) row-major, or stored transposed (K,M) when trans_a; B is (K,N) row-major, or
 * stored transposed (N,K) when trans_b; bf16 operands, FP32 accumulation. M, N multiples of 64, K a multiple of 32.
 * epilogue: 0 C f32 = acc (splits > 1 splits K over `splits` CTAs, reduced in fixed order through split_ws of
 * splits*M*N floats); 1 C f32 = acc + bias; 2 C bf16 = relu(acc + bias); 3 C bf16 = acc + bias;
 * 4 C bf16 = (mask > 0) ? acc : 0 with mask (M,N) bf16. */
int lddmm_bf16_gemm(int trans_a, int trans_b, int epilogue, int64_t M, int64_t N, int64_t K, const void* A,
                    const void* B, const float* bias, const void* mask, void* C, int splits, float* split_ws,
                    size_t split_ws_bytes, lddmm_stream_t stream);

/* db(N) = column sums of dy (M,N) bf16, FP32, fixed order. With a workspace ws of at least ceil(M/256)*N floats
 * the rows are split over the whole GPU (two stages, still fixed order); ws = NULL sums with N/32 CTAs. */
int lddmm_bf16_colsum(const void* dy, int64_t M, int64_t N, float* db, float* ws, size_t ws_bytes,
                      lddmm_stream_t stream);

/* Squared-error gradient of the first nout columns of y (M,N) f32 against target (M,nout) f32 for rows < valid:
 * dy (M,N) bf16 = 2 w (y - target) there and 0 elsewhere; row_loss (M) f32 = per-row squared errors. */
int lddmm_mse_grad(const float* y, int64_t M, int64_t N, const float* target, int64_t nout, int64_t valid, float w,
                   void* dy, float* row_loss, lddmm_stream_t stream);

/* Adam step on FP32 master weights (step >= 1, bias-corrected), writing the bf16 copy param_bf16 (may be NULL). */
int lddmm_adam_step(float* param, const float* grad, float* m1, float* m2, void* param_bf16, int64_t count, float lr,
                    float beta1, float beta2, float eps, int64_t step, float weight_decay, lddmm_stream_t stream);

/* disp(n,3) = tgt[argmin_l |src_k - tgt_l|] - src_k: nearest-target displacement of every source point. */
int lddmm_nearest_displacement(const double* src, int64_t n, const double* tgt, int64_t m, double* disp,
                               lddmm_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Optimiser: the L-BFGS search direction (replaces the two-loop recursion of base/bfgs.py:183-198).
 * q(n) = H g for the m stored pairs (s_k, y_k), k = 0 oldest .. m-1 newest: rho_k = 1/(y_k.s_k), the initial
 * scaling (s_{m-1}.y_{m-1})/(y_{m-1}.y_{m-1}) (1 when below 1e-10), all in FP64 and in one launch (one CTA, fixed
 * reduction order). s and y are HOST arrays of m device pointers to n doubles each; g and q are device arrays of n
 * doubles (q may not alias g, s or y). 1 <= m <= LDDMM_LBFGS_MAX_PAIRS. Meant for the small and medium controls
 * of the coarse levels (n up to ~1e5), where the recursion from the host costs more than the shooting. */
#define LDDMM_LBFGS_MAX_PAIRS 64
int lddmm_lbfgs_direction(const double* const* s, const double* const* y, int m, const double* g, int64_t n,
                          double* q, lddmm_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* LDDMM_B200_H */
