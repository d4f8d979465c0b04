// cg.cu -- conjugate-gradient cone-beam reconstruction on sm_100a.
//
// Restates rtk::ConjugateGradientConeBeamReconstructionFilter
// (include/rtkConjugateGradientConeBeamReconstructionFilter.hxx:192-305),
// rtk::ReconstructionConjugateGradientOperator
// (include/rtkReconstructionConjugateGradientOperator.hxx:192-286) and
// rtk::ConjugateGradientImageFilter::GenerateData
// (include/rtkConjugateGradientImageFilter.hxx:108-258); replaces
// CUDA_conjugate_gradient (src/rtkCudaConjugateGradientImageFilter.cu:80-166),
// which calls cuBLAS with a handle per call and round-trips alpha and beta to
// the host.
//
// A plan owns every device buffer, so one iteration allocates nothing and is
// captured once as a CUDA graph.  Operator: A x = BP(W .* FP(x)) + tikhonov x
// with the Joseph pair, W the displaced-detector weights of the input weights
// (no padding).  Vectors are FP32; the dot products (deterministic two-pass
// reductions), alpha and beta are FP64 and never leave the device.
#include "rtkb_elem.cuh"
#include "rtkb_joseph.h"

#include "rtkb_backproject.h"

#include <cfloat>
#include <cstring>
#include <vector>

struct rtkb_cg
{
  rtkb_geometry *          g = nullptr;  // private copy of the geometry
  rtkb_image_desc          vol{}, proj{};
  rtkb::JosephArgs         args{};
  float                    tikhonov = 0.f;
  float                    gamma = 0.f; // Laplacian regularisation weight (RTK's SetGamma)
  bool                     use_graph = true;
  bool                     bf16 = false;  // R, P, AP and tmp stored as bfloat16 (FP32 arithmetic)
  bool                     bf16p = false; // P and tmp stored as bfloat16; R, AP and x FP32
  long long                nvox = 0, npix = 0;
  void *                   mem = nullptr; // one device allocation for everything below
  rtkb::RayProj *          tab = nullptr;
  float *                  W = nullptr; // weights (null: all ones)
  float *                  tmp = nullptr;
  float *                  R = nullptr; // R, P, AP hold bfloat16 values in a BF16 plan
  float *                  P = nullptr;
  float *                  AP = nullptr;
  void *                   scratch = nullptr; // projector scratch (copies and accumulators of the volume)
  double *                 scal = nullptr; // rr, rr0, alpha, beta, pAp
  double *                 partial = nullptr;
  float *                  x = nullptr; // the iterate (caller's buffer)
  cudaStream_t             cap = nullptr; // private stream the iteration graph is captured on
  cudaGraph_t              graph = nullptr;
  cudaGraphExec_t          exec = nullptr;
  int                      iterations = 0;
  // flexible PCG with a learned preconditioner (optional)
  rtkb_unet *              net = nullptr;
  void *                   pmem = nullptr; // Z and the second partial-sum buffer
  float *                  Z = nullptr;
  double *                 partial2 = nullptr;
  int                      m = 0;              // directions kept for re-orthogonalisation
  float *                  Ph = nullptr;       // m previous directions
  float *                  APh = nullptr;      // A times each of them
  double *                 hist = nullptr;     // [m] <p_j, A p_j>, [m] beta_j, [1] slot counter
  double *                 mpartial = nullptr; // [m][kRedBlocks] partial dot products
  bool                     pcg_active = false;
  int                      fallback_iteration = -1;
  double                   rr_best = 0.;
  int                      stall = 0;
  cudaGraph_t              graph_p = nullptr;
  cudaGraphExec_t          exec_p = nullptr;
  // support mask (SetSupportMask): caller's volume, and the masked operator input
  const float *            mask = nullptr;
  float *                  Mx = nullptr;
  // voxel-based back projector (BP_VOXELBASED) reading tmp, instead of Joseph's
  bool                     voxel_bp = false;
  rtkb::VoxelBackprojector vbp{};
};

namespace rtkb
{
cudaError_t unet_apply(rtkb_unet * u, const float * in, float * out, cudaStream_t st);
bool        unet_reserved_for(const rtkb_unet * u, int nx, int ny, int nz);
} // namespace rtkb

namespace
{
using rtkb::Elem;
using rtkb::ld_elem;
using rtkb::st_elem;

constexpr int kRedBlocks = 148 * 4;
constexpr int kRedThreads = 256;
enum
{
  S_RR = 0,
  S_RR0 = 1,
  S_ALPHA = 2,
  S_BETA = 3,
  S_PAP = 4
};
// Flexible PCG patience: fall back to plain CG when ||r|| has not improved on
// its best value for this many consecutive iterations.
constexpr int kPcgPatience = 2;

__device__ __forceinline__ double
block_sum(double v)
{
  __shared__ double sh[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRedThreads / 32; w++)
      s += sh[w];
  return s;
}

// partial[b] = sum over block b's fixed slice of a[i] * b[i] (FP64)
template <typename SA, typename SB = SA>
__global__ void __launch_bounds__(kRedThreads)
dot_partial_kernel(const SA * __restrict__ a, const SB * __restrict__ b, long long n, double * partial)
{
  double s = 0.;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)kRedBlocks * kRedThreads)
    s = fma((double)ld_elem(a, i), (double)ld_elem(b, i), s);
  s = block_sum(s);
  if (threadIdx.x == 0)
    partial[blockIdx.x] = s;
}

// x += alpha p; r -= alpha ap; partial of <r, r> (of r as stored); r and ap
// stored as SR, p as SP
template <typename SR, typename SP = SR>
__global__ void __launch_bounds__(kRedThreads)
update_xr_kernel(float * __restrict__ x, SR * __restrict__ r, const SP * __restrict__ p, const SR * __restrict__ ap,
                 long long n, const double * __restrict__ scal, double * partial)
{
  const double alpha = scal[S_ALPHA];
  const float  af = (float)alpha;
  double       s = 0.;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)kRedBlocks * kRedThreads)
  {
    x[i] = fmaf(af, ld_elem(p, i), x[i]);
    st_elem(r, i, fmaf(-af, ld_elem(ap, i), ld_elem(r, i)));
    const float ri = ld_elem(r, i);
    s = fma((double)ri, (double)ri, s);
  }
  s = block_sum(s);
  if (threadIdx.x == 0)
    partial[blockIdx.x] = s;
}

__device__ __forceinline__ double
sum_partials(const double * partial)
{
  // one warp, fixed order
  double s = 0.;
  for (int i = threadIdx.x; i < kRedBlocks; i += 32)
    s += partial[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// alpha = rr / (pAp + eps)
__global__ void
finalize_alpha_kernel(const double * partial, double * scal)
{
  const double pap = sum_partials(partial);
  if (threadIdx.x == 0)
  {
    scal[S_PAP] = pap;
    scal[S_ALPHA] = scal[S_RR] / (pap + DBL_MIN);
  }
}

// beta = rr_new / (rr + eps); rr = rr_new
__global__ void
finalize_beta_kernel(const double * partial, double * scal)
{
  const double rr = sum_partials(partial);
  if (threadIdx.x == 0)
  {
    scal[S_BETA] = rr / (scal[S_RR] + DBL_MIN);
    scal[S_RR] = rr;
  }
}

// rr = rr0 = sum of partials (start)
__global__ void
finalize_start_kernel(const double * partial, double * scal)
{
  const double rr = sum_partials(partial);
  if (threadIdx.x == 0)
  {
    scal[S_RR] = rr;
    scal[S_RR0] = rr;
  }
}

// p = r + beta p
template <typename SP, typename SR = SP>
__global__ void __launch_bounds__(256)
update_p_kernel(SP * __restrict__ p, const SR * __restrict__ r, long long n, const double * __restrict__ scal)
{
  const float beta = (float)scal[S_BETA];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    st_elem(p, i, fmaf(beta, ld_elem(p, i), ld_elem(r, i)));
}

// r = r - ap; p = r (start: R0 = B - A x0)
template <typename SR, typename SP = SR>
__global__ void __launch_bounds__(256)
start_rp_kernel(SR * __restrict__ r, SP * __restrict__ p, const SR * __restrict__ ap, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const float v = ld_elem(r, i) - ld_elem(ap, i);
    st_elem(r, i, v);
    st_elem(p, i, v);
  }
}

// out = a .* b (b may be null: copy), stored as TO
template <typename TO>
__global__ void __launch_bounds__(256)
mul_kernel(TO * __restrict__ out, const float * __restrict__ a, const float * __restrict__ b, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    st_elem(out, i, b ? a[i] * b[i] : a[i]);
}

// x = x .* m, in place
__global__ void __launch_bounds__(256)
mask_inplace_kernel(float * x, const float * __restrict__ m, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = x[i] * m[i];
}

__global__ void __launch_bounds__(256)
fill_kernel(float * __restrict__ out, float v, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = v;
}

// partial[b] = <a1, b1>, partial2[b] = <a2, b2> over block b's slice (FP64)
__global__ void __launch_bounds__(kRedThreads)
dot2_partial_kernel(const float * __restrict__ a1, const float * __restrict__ b1, const float * __restrict__ a2,
                    const float * __restrict__ b2, long long n, double * partial, double * partial2)
{
  double s1 = 0., s2 = 0.;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)kRedBlocks * kRedThreads)
  {
    s1 = fma((double)a1[i], (double)b1[i], s1);
    s2 = fma((double)a2[i], (double)b2[i], s2);
  }
  s1 = block_sum(s1);
  __syncthreads();
  s2 = block_sum(s2);
  if (threadIdx.x == 0)
  {
    partial[blockIdx.x] = s1;
    partial2[blockIdx.x] = s2;
  }
}

// flexible PCG: alpha = <p, r> / (<p, Ap> + eps)
__global__ void
finalize_alpha_pcg_kernel(const double * partial, const double * partial2, double * scal)
{
  const double pap = sum_partials(partial);
  const double pr = sum_partials(partial2);
  if (threadIdx.x == 0)
  {
    scal[S_PAP] = pap;
    scal[S_ALPHA] = pr / (pap + DBL_MIN);
  }
}

// rr = <r, r> (no beta: the PCG direction update comes after the preconditioner)
__global__ void
finalize_rr_kernel(const double * partial, double * scal)
{
  const double rr = sum_partials(partial);
  if (threadIdx.x == 0)
    scal[S_RR] = rr;
}

// Truncated flexible CG keeps the last m directions p_j, A p_j and <p_j, A p_j>
// in a ring; slot = counter mod m.  Store the current direction there.
constexpr int kMaxHistory = 16;
__global__ void __launch_bounds__(256)
store_direction_kernel(const float * __restrict__ p, const float * __restrict__ ap, float * __restrict__ ph,
                       float * __restrict__ aph, long long n, int m, const double * __restrict__ scal,
                       double * __restrict__ hist)
{
  const int slot = (int)hist[2 * m] % m;
  float *   dp = ph + (size_t)slot * n;
  float *   dap = aph + (size_t)slot * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    dp[i] = p[i];
    dap[i] = ap[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    hist[slot] = scal[S_PAP];
}

__global__ void
advance_slot_kernel(double * hist, int m)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
    hist[2 * m] += 1.;
}

// mpartial[j][b] = <z, A p_j> over block b's slice, j < m (FP64)
__global__ void __launch_bounds__(kRedThreads)
multi_dot_kernel(const float * __restrict__ z, const float * __restrict__ aph, long long n, int m,
                 double * __restrict__ mpartial)
{
  double s[kMaxHistory];
#pragma unroll
  for (int j = 0; j < kMaxHistory; j++)
    s[j] = 0.;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)kRedBlocks * kRedThreads)
  {
    const double zi = z[i];
#pragma unroll
    for (int j = 0; j < kMaxHistory; j++)
      if (j < m)
        s[j] = fma(zi, (double)aph[(size_t)j * n + i], s[j]);
  }
#pragma unroll 1
  for (int j = 0; j < m; j++)
  {
    const double t = block_sum(s[j]);
    if (threadIdx.x == 0)
      mpartial[(size_t)j * kRedBlocks + blockIdx.x] = t;
    __syncthreads();
  }
}

// beta_j = -<z, A p_j> / <p_j, A p_j> (0 for empty slots): A-orthogonalises the
// new direction against the kept ones (Notay's truncated flexible CG)
__global__ void
finalize_betas_kernel(const double * __restrict__ mpartial, int m, double * __restrict__ hist)
{
  for (int j = 0; j < m; j++)
  {
    const double zap = sum_partials(mpartial + (size_t)j * kRedBlocks);
    if (threadIdx.x == 0)
      hist[m + j] = hist[j] > 0. ? -zap / hist[j] : 0.;
  }
}

// p = z + sum_j beta_j p_j
__global__ void __launch_bounds__(256)
update_p_multi_kernel(float * __restrict__ p, const float * __restrict__ z, const float * __restrict__ ph, long long n,
                      int m, const double * __restrict__ hist)
{
  float b[kMaxHistory];
#pragma unroll
  for (int j = 0; j < kMaxHistory; j++)
    b[j] = j < m ? (float)hist[m + j] : 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    float v = z[i];
#pragma unroll
    for (int j = 0; j < kMaxHistory; j++)
      if (j < m)
        v = fmaf(b[j], ph[(size_t)j * n + i], v);
    p[i] = v;
  }
}

unsigned
grid_for(long long n)
{
  return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
}

// RTK's LaplacianImageFilter (include/rtkLaplacianImageFilter.hxx: backward-
// difference divergence of the forward-difference gradient, zero-flux
// Neumann boundary, spacing-scaled): per axis, the sum over the existing
// neighbours of (x_nb - x_i) * w_axis with w = 1 / spacing^2.
// out = scale * Laplacian(x), or out += scale * Laplacian(x) when add.
// Threads along x, blocks over (x tiles, y, z), striding past the grid's
// limits: no per-voxel division.
template <typename TI, typename TO>
__global__ void __launch_bounds__(128)
laplacian_kernel(const TI * __restrict__ x, TO * out, int nx, int ny, int nz, float wx, float wy, float wz,
                 float scale, bool add)
{
  const long long sxy = (long long)nx * ny;
  const int       ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= nx)
    return;
  for (int iz = blockIdx.z; iz < nz; iz += gridDim.z)
    for (int iy = blockIdx.y; iy < ny; iy += gridDim.y)
    {
      const long long i = (long long)iz * sxy + (long long)iy * nx + ix;
      const float c = ld_elem(x, i);
      float       lx = 0.f, ly = 0.f, lz = 0.f;
      if (ix + 1 < nx)
        lx += ld_elem(x, i + 1) - c;
      if (ix > 0)
        lx += ld_elem(x, i - 1) - c;
      if (iy + 1 < ny)
        ly += ld_elem(x, i + nx) - c;
      if (iy > 0)
        ly += ld_elem(x, i - nx) - c;
      if (iz + 1 < nz)
        lz += ld_elem(x, i + sxy) - c;
      if (iz > 0)
        lz += ld_elem(x, i - sxy) - c;
      const float l = fmaf(lx, wx, fmaf(ly, wy, lz * wz));
      st_elem(out, i, add ? fmaf(scale, l, ld_elem(out, i)) : scale * l);
    }
}

template <typename TI, typename TO>
cudaError_t
laplacian_launch(const rtkb_image_desc & v, const TI * x, TO * out, float scale, bool add, cudaStream_t st)
{
  const dim3 grid((unsigned)((v.size[0] + 127) / 128), (unsigned)std::min(v.size[1], 65535),
                  (unsigned)std::min(v.size[2], 65535));
  laplacian_kernel<TI, TO><<<grid, 128, 0, st>>>(
    x, out, v.size[0], v.size[1], v.size[2], (float)(1. / (v.spacing[0] * v.spacing[0])),
    (float)(1. / (v.spacing[1] * v.spacing[1])), (float)(1. / (v.spacing[2] * v.spacing[2])), scale, add);
  return cudaGetLastError();
}

// storage of the projection-domain temporary (tmp), of the direction P, and
// of R and AP: all FP32 (storage 0); all BF16 (storage 1); P and tmp BF16
// with R, AP and the iterate FP32 (storage 2)
Elem
storage(const rtkb_cg * c)
{
  return (c->bf16 || c->bf16p) ? Elem::BF16 : Elem::F32;
}

Elem
pstore(const rtkb_cg * c)
{
  return (c->bf16 || c->bf16p) ? Elem::BF16 : Elem::F32;
}

Elem
rstore(const rtkb_cg * c)
{
  return c->bf16 ? Elem::BF16 : Elem::F32;
}

template <typename S>
S *
as(float * p)
{
  return reinterpret_cast<S *>(p);
}

cudaError_t add_laplacian(rtkb_cg * c, const void * in, Elem ie, void * out, Elem oe, cudaStream_t st);

__global__ void
scale_kernel(float * __restrict__ out, const float * __restrict__ in, float s, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = s * in[i];
}

// out = BP_voxel(tmp) + tikhonov * x (x may be null: no Tikhonov term); FP32 plans
cudaError_t
voxel_bp_into(rtkb_cg * c, const float * x, float * out, cudaStream_t st)
{
  if (x)
    scale_kernel<<<grid_for(c->nvox), 256, 0, st>>>(out, x, c->tikhonov, c->nvox);
  else
  {
    const cudaError_t e = cudaMemsetAsync(out, 0, (size_t)c->nvox * sizeof(float), st);
    if (e != cudaSuccess)
      return e;
  }
  const int rc = rtkb::voxel_backprojector_launch(c->vbp, out, out, st);
  return rc == RTKB_OK ? cudaGetLastError() : cudaErrorLaunchFailure;
}

// out = A in (uses tmp and the projector scratch); in and out have storage
// ie and oe, tmp the plan's storage
cudaError_t
apply_A(rtkb_cg * c, const void * in, Elem ie, void * out, Elem oe, cudaStream_t st)
{
  if (c->mask)
  {
    // with a support mask M (FP32 plans): A x = M .* (BP(W .* FP(M .* x)) + gamma (-Laplacian(M .* x)) + tau M .* x)
    // (ReconstructionConjugateGradientOperator, include/rtkReconstructionConjugateGradientOperator.hxx:203-262)
    mul_kernel<float><<<grid_for(c->nvox), 256, 0, st>>>(c->Mx, static_cast<const float *>(in), c->mask, c->nvox);
    in = c->Mx;
    ie = Elem::F32;
  }
  cudaError_t e = rtkb::joseph_forward_launch(c->args, in, ie, c->scratch, nullptr, c->tmp, storage(c), c->W, st);
  if (e != cudaSuccess)
    return e;
  if (c->voxel_bp)
    e = voxel_bp_into(c, c->tikhonov != 0.f ? static_cast<const float *>(in) : nullptr, static_cast<float *>(out), st);
  else
    e = rtkb::joseph_back_launch(c->args, c->tmp, storage(c), c->scratch, nullptr, out, oe,
                                 c->tikhonov != 0.f ? in : nullptr, ie, c->tikhonov, st);
  if (e != cudaSuccess)
    return e;
  if (c->gamma != 0.f)
    e = add_laplacian(c, in, ie, out, oe, st);
  if (e == cudaSuccess && c->mask)
  {
    mask_inplace_kernel<<<grid_for(c->nvox), 256, 0, st>>>(static_cast<float *>(out), c->mask, c->nvox);
    e = cudaGetLastError();
  }
  return e;
}

// out += gamma * (-Laplacian(in))
cudaError_t
add_laplacian(rtkb_cg * c, const void * in, Elem ie, void * out, Elem oe, cudaStream_t st)
{
  // + gamma * (-Laplacian(in)) (ReconstructionConjugateGradientOperator, include/rtkReconstructionConjugateGradientOperator.hxx:294-311)
  using B = __nv_bfloat16;
  if (ie == Elem::BF16)
    return oe == Elem::BF16 ? laplacian_launch(c->vol, static_cast<const B *>(in), static_cast<B *>(out), -c->gamma, true, st)
                            : laplacian_launch(c->vol, static_cast<const B *>(in), static_cast<float *>(out), -c->gamma, true, st);
  return oe == Elem::BF16 ? laplacian_launch(c->vol, static_cast<const float *>(in), static_cast<B *>(out), -c->gamma, true, st)
                          : laplacian_launch(c->vol, static_cast<const float *>(in), static_cast<float *>(out), -c->gamma, true, st);
}

template <typename SR, typename SP>
cudaError_t
enqueue_iteration_t(rtkb_cg * c, cudaStream_t st)
{
  SP *        P = as<SP>(c->P);
  SR *        AP = as<SR>(c->AP);
  SR *        R = as<SR>(c->R);
  cudaError_t e = apply_A(c, P, pstore(c), AP, rstore(c), st);
  if (e != cudaSuccess)
    return e;
  dot_partial_kernel<SP, SR><<<kRedBlocks, kRedThreads, 0, st>>>(P, AP, c->nvox, c->partial);
  finalize_alpha_kernel<<<1, 32, 0, st>>>(c->partial, c->scal);
  update_xr_kernel<SR, SP><<<kRedBlocks, kRedThreads, 0, st>>>(c->x, R, P, AP, c->nvox, c->scal, c->partial);
  finalize_beta_kernel<<<1, 32, 0, st>>>(c->partial, c->scal);
  update_p_kernel<SP, SR><<<grid_for(c->nvox), 256, 0, st>>>(P, R, c->nvox, c->scal);
  return cudaGetLastError();
}

cudaError_t
enqueue_iteration(rtkb_cg * c, cudaStream_t st)
{
  using B = __nv_bfloat16;
  if (c->bf16)
    return enqueue_iteration_t<B, B>(c, st);
  return c->bf16p ? enqueue_iteration_t<float, B>(c, st) : enqueue_iteration_t<float, float>(c, st);
}

// One truncated flexible-PCG iteration: Ap; alpha = <p,r>/<p,Ap>;
// x += alpha p; r -= alpha Ap; keep (p, Ap, <p,Ap>); z = M(r);
// p = z - sum_j <z,Ap_j>/<p_j,Ap_j> p_j over the kept directions.
cudaError_t
enqueue_pcg_iteration(rtkb_cg * c, cudaStream_t st)
{
  cudaError_t e = apply_A(c, c->P, Elem::F32, c->AP, Elem::F32, st);
  if (e != cudaSuccess)
    return e;
  dot2_partial_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(c->P, c->AP, c->P, c->R, c->nvox, c->partial, c->partial2);
  finalize_alpha_pcg_kernel<<<1, 32, 0, st>>>(c->partial, c->partial2, c->scal);
  update_xr_kernel<float><<<kRedBlocks, kRedThreads, 0, st>>>(c->x, c->R, c->P, c->AP, c->nvox, c->scal, c->partial);
  finalize_rr_kernel<<<1, 32, 0, st>>>(c->partial, c->scal);
  store_direction_kernel<<<grid_for(c->nvox), 256, 0, st>>>(c->P, c->AP, c->Ph, c->APh, c->nvox, c->m, c->scal,
                                                             c->hist);
  advance_slot_kernel<<<1, 32, 0, st>>>(c->hist, c->m);
  e = rtkb::unet_apply(c->net, c->R, c->Z, st);
  if (e != cudaSuccess)
    return e;
  multi_dot_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(c->Z, c->APh, c->nvox, c->m, c->mpartial);
  finalize_betas_kernel<<<1, 32, 0, st>>>(c->mpartial, c->m, c->hist);
  update_p_multi_kernel<<<grid_for(c->nvox), 256, 0, st>>>(c->P, c->Z, c->Ph, c->nvox, c->m, c->hist);
  return cudaGetLastError();
}

cudaError_t
capture(rtkb_cg * c, bool pcg, cudaGraph_t * graph, cudaGraphExec_t * exec)
{
  cudaError_t e = cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess)
  {
    cudaError_t ei = pcg ? enqueue_pcg_iteration(c, c->cap) : enqueue_iteration(c, c->cap);
    e = cudaStreamEndCapture(c->cap, graph);
    if (e == cudaSuccess)
      e = ei;
  }
  if (e == cudaSuccess)
    e = cudaGraphInstantiate(exec, *graph, 0);
  return e;
}

void
drop_graphs(rtkb_cg * c)
{
  if (c->exec)
    cudaGraphExecDestroy(c->exec);
  if (c->graph)
    cudaGraphDestroy(c->graph);
  if (c->exec_p)
    cudaGraphExecDestroy(c->exec_p);
  if (c->graph_p)
    cudaGraphDestroy(c->graph_p);
  c->exec = nullptr;
  c->graph = nullptr;
  c->exec_p = nullptr;
  c->graph_p = nullptr;
}

void
release(rtkb_cg * c)
{
  if (!c)
    return;
  drop_graphs(c);
  if (c->Mx)
    cudaFree(c->Mx);
  if (c->pmem)
    cudaFree(c->pmem);
  if (c->mem)
    cudaFree(c->mem);
  if (c->cap)
    cudaStreamDestroy(c->cap);
  delete c->g;
  delete c;
}

} // namespace

extern "C" int
rtkb_cg_create(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
               const rtkb_cg_params * params, rtkb_cg ** out)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null plan pointer");
  *out = nullptr;
  int rc = joseph_check(g, vol, proj);
  if (rc != RTKB_OK)
    return rc;
  rtkb_cg * c = nullptr;
  try
  {
    c = new rtkb_cg();
    c->g = new rtkb_geometry(*g);
    c->vol = *vol;
    c->proj = *proj;
    c->tikhonov = params ? (float)params->tikhonov : 0.f;
    c->gamma = params ? (float)params->gamma : 0.f;
    c->use_graph = params ? params->use_cuda_graph != 0 : true;
    c->bf16 = params ? params->storage == 1 : false;
    c->bf16p = params ? params->storage == 2 : false;
    if (params && (params->storage < 0 || params->storage > 2))
    {
      release(c);
      return fail(RTKB_ERR_INVALID_ARGUMENT, "storage must be 0 (FP32), 1 or 2 (BF16 variants)");
    }
    // RTK's BackProjectionType: BP_VOXELBASED 0 (its default), BP_JOSEPH 1, BP_CUDAVOXELBASED 2
    const int bpt = params ? params->backprojector : 0;
    if (bpt < 0 || bpt > 2)
    {
      release(c);
      return fail(RTKB_ERR_UNSUPPORTED, "back projector: BP_VOXELBASED (0), BP_JOSEPH (1) or BP_CUDAVOXELBASED (2)");
    }
    c->voxel_bp = bpt != 1;
    if (c->voxel_bp && (c->bf16 || c->bf16p || g->g.radius_cylindrical != 0.))
    {
      release(c);
      return fail(RTKB_ERR_UNSUPPORTED, "the voxel-based back projector in CG needs FP32 storage and a flat panel");
    }
    c->nvox = num_pixels(*vol);
    c->npix = num_pixels(*proj);
    std::vector<RayProj> tab;
    std::vector<CylProj> cyl;
    rc = joseph_tables(g->g, *vol, *proj, tab, &cyl);
    if (rc != RTKB_OK)
    {
      release(c);
      return rc;
    }
    auto         up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t tb = joseph_table_bytes(tab, cyl), pb = up((size_t)c->npix * 4), vb = up((size_t)c->nvox * 4);
    const size_t sb = up(8 * sizeof(double)), rb = up(kRedBlocks * sizeof(double));
    const size_t fb = up(std::max(joseph_forward_scratch_bytes(c->nvox), joseph_back_scratch_bytes(c->nvox)));
    const size_t xb = c->voxel_bp ? voxel_backprojector_bytes(proj->size[2]) : 0;
    const size_t total = tb + 2 * pb + 3 * vb + sb + rb + fb + xb;
    cudaError_t  e = cudaMalloc(&c->mem, total);
    if (e == cudaSuccess && c->use_graph)
      e = cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
      release(c);
      return cuda_fail(e, "cudaMalloc (CG plan)");
    }
    char * m = static_cast<char *>(c->mem);
    c->tab = reinterpret_cast<RayProj *>(m);
    m += tb;
    c->W = reinterpret_cast<float *>(m);
    m += pb;
    c->tmp = reinterpret_cast<float *>(m);
    m += pb;
    c->R = reinterpret_cast<float *>(m);
    m += vb;
    c->P = reinterpret_cast<float *>(m);
    m += vb;
    c->AP = reinterpret_cast<float *>(m);
    m += vb;
    c->scal = reinterpret_cast<double *>(m);
    m += sb;
    c->partial = reinterpret_cast<double *>(m);
    m += rb;
    c->scratch = m;
    m += fb;
    if (c->voxel_bp)
    {
      rc = voxel_backprojector_create(g, *vol, *proj, c->tmp, m, c->vbp);
      if (rc != RTKB_OK)
      {
        release(c);
        return rc;
      }
    }
    joseph_args(c->args, *vol, *proj, nullptr);
    e = joseph_upload_tables(tab, cyl, g->g.radius_cylindrical, c->tab, c->args, nullptr);
    if (e == cudaSuccess)
      e = cudaMemset(c->scal, 0, sb);
    if (e == cudaSuccess)
    {
      fill_kernel<<<grid_for(c->npix), 256>>>(c->W, 1.f, c->npix); // W = 1 until rtkb_cg_start sets it
      e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess)
    {
      release(c);
      return cuda_fail(e, "CG plan upload");
    }
    *out = c;
    return RTKB_OK;
  }
  catch (...)
  {
    release(c);
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

namespace
{
// Shared tail of the two starts: R holds b on entry; R = b - A x0, P = R (or
// M(R) with a preconditioner), rr; then the iteration graphs are captured.
int
start_from_rhs(rtkb_cg * c, cudaStream_t st)
{
  using namespace rtkb;
  cudaError_t e = apply_A(c, c->x, Elem::F32, c->AP, rstore(c), st);
  if (e != cudaSuccess)
    return cuda_fail(e, "CG start");
  if (c->bf16)
  {
    using B = __nv_bfloat16;
    start_rp_kernel<B><<<grid_for(c->nvox), 256, 0, st>>>(as<B>(c->R), as<B>(c->P), as<B>(c->AP), c->nvox);
    dot_partial_kernel<B><<<kRedBlocks, kRedThreads, 0, st>>>(as<B>(c->R), as<B>(c->R), c->nvox, c->partial);
  }
  else if (c->bf16p)
  {
    using B = __nv_bfloat16;
    start_rp_kernel<float, B><<<grid_for(c->nvox), 256, 0, st>>>(c->R, as<B>(c->P), c->AP, c->nvox);
    dot_partial_kernel<float><<<kRedBlocks, kRedThreads, 0, st>>>(c->R, c->R, c->nvox, c->partial);
  }
  else
  {
    start_rp_kernel<float><<<grid_for(c->nvox), 256, 0, st>>>(c->R, c->P, c->AP, c->nvox);
    dot_partial_kernel<float><<<kRedBlocks, kRedThreads, 0, st>>>(c->R, c->R, c->nvox, c->partial);
  }
  finalize_start_kernel<<<1, 32, 0, st>>>(c->partial, c->scal);
  RTKB_CUDA_TRY(cudaGetLastError());
  if (c->pcg_active)
  {
    // empty direction history; z0 = M(r0), p0 = z0 (run eagerly once, before any capture)
    RTKB_CUDA_TRY(cudaMemsetAsync(c->hist, 0, (2 * c->m + 1) * sizeof(double), st));
    RTKB_CUDA_TRY(unet_apply(c->net, c->R, c->Z, st));
    mul_kernel<float><<<grid_for(c->nvox), 256, 0, st>>>(c->P, c->Z, nullptr, c->nvox);
    RTKB_CUDA_TRY(cudaGetLastError());
    double h[2] = { 0., 0. };
    RTKB_CUDA_TRY(cudaMemcpyAsync(h, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    RTKB_CUDA_TRY(cudaStreamSynchronize(st));
    c->rr_best = h[S_RR];
  }
  if (c->use_graph)
  {
    // capture one iteration once on the plan's private stream (the caller's
    // may be the legacy default stream, which cannot be captured); later
    // iterations replay it on the caller's stream
    e = capture(c, false, &c->graph, &c->exec);
    if (e == cudaSuccess && c->pcg_active)
      e = capture(c, true, &c->graph_p, &c->exec_p);
    if (e != cudaSuccess)
      return cuda_fail(e, "CG graph capture");
  }
  return RTKB_OK;
}

void
reset_run(rtkb_cg * c, float * d_x)
{
  drop_graphs(c);
  c->x = d_x;
  c->iterations = 0;
  c->pcg_active = c->net != nullptr;
  c->fallback_iteration = -1;
  c->stall = 0;
}
} // namespace

namespace
{
// W = displaced-detector weights (no padding) of the input weights (ones by
// default), then out = BP(W .* p) in the storage type oe.
int
weights_and_rhs(rtkb_cg * c, const float * d_proj, const float * d_weights, int displaced_detector, void * out,
                rtkb::Elem oe, cudaStream_t st)
{
  using namespace rtkb;
  const bool have_w = d_weights != nullptr;
  if (displaced_detector)
  {
    if (!have_w)
      fill_kernel<<<grid_for(c->npix), 256, 0, st>>>(c->tmp, 1.f, c->npix);
    const int rc = rtkb_displaced_detector(c->g, &c->proj, 0, have_w ? d_weights : c->tmp, c->W, st);
    if (rc != RTKB_OK)
      return rc;
  }
  else if (have_w)
    RTKB_CUDA_TRY(cudaMemcpyAsync(c->W, d_weights, (size_t)c->npix * 4, cudaMemcpyDeviceToDevice, st));
  else
    fill_kernel<<<grid_for(c->npix), 256, 0, st>>>(c->W, 1.f, c->npix);
  // tmp = W .* p in the plan's storage
  if (storage(c) == Elem::BF16)
    mul_kernel<__nv_bfloat16><<<grid_for(c->npix), 256, 0, st>>>(as<__nv_bfloat16>(c->tmp), d_proj, c->W, c->npix);
  else
    mul_kernel<float><<<grid_for(c->npix), 256, 0, st>>>(c->tmp, d_proj, c->W, c->npix);
  cudaError_t e = c->voxel_bp ? voxel_bp_into(c, nullptr, static_cast<float *>(out), st)
                              : joseph_back_launch(c->args, c->tmp, storage(c), c->scratch, nullptr, out, oe, nullptr,
                                                   Elem::F32, 0.f, st);
  if (e == cudaSuccess && c->mask)
  {
    // b = M .* BP(W .* p) (ConjugateGradientConeBeamReconstructionFilter with a support mask)
    mask_inplace_kernel<<<grid_for(c->nvox), 256, 0, st>>>(static_cast<float *>(out), c->mask, c->nvox);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "CG right-hand side");
}
} // namespace

namespace rtkb
{
int
cg_rhs(rtkb_cg * c, const float * d_proj, const float * d_weights, int displaced_detector, float * d_b,
       cudaStream_t st)
{
  if (!c || !d_proj || !d_b)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  return weights_and_rhs(c, d_proj, d_weights, displaced_detector, d_b, Elem::F32, st);
}
} // namespace rtkb

extern "C" int
rtkb_cg_start(rtkb_cg * c, const float * d_proj, const float * d_weights, int displaced_detector, float * d_x,
              void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c || !d_proj || !d_x)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  reset_run(c, d_x);
  // R = b = BP(W .* p)
  const int rc = weights_and_rhs(c, d_proj, d_weights, displaced_detector, c->R, rstore(c), st);
  if (rc != RTKB_OK)
    return rc;
  return start_from_rhs(c, st);
}

extern "C" int
rtkb_cg_start_rhs(rtkb_cg * c, const float * d_b, float * d_x, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c || !d_b || !d_x)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  reset_run(c, d_x);
  if (c->bf16)
    mul_kernel<__nv_bfloat16><<<grid_for(c->nvox), 256, 0, st>>>(as<__nv_bfloat16>(c->R), d_b, nullptr, c->nvox);
  else
    RTKB_CUDA_TRY(cudaMemcpyAsync(c->R, d_b, (size_t)c->nvox * 4, cudaMemcpyDeviceToDevice, st));
  RTKB_CUDA_TRY(cudaGetLastError());
  return start_from_rhs(c, st);
}

extern "C" int
rtkb_cg_iterate(rtkb_cg * c, int n, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c || !c->x || n < 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "CG plan not started");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int i = 0; i < n; i++)
  {
    if (c->pcg_active)
    {
      cudaError_t e = c->exec_p ? cudaGraphLaunch(c->exec_p, st) : enqueue_pcg_iteration(c, st);
      if (e != cudaSuccess)
        return cuda_fail(e, "PCG iteration");
      c->iterations++;
      // the true normal-equation residual judges the preconditioner: when
      // ||r|| stops improving, continue as plain CG from the current iterate
      double rr = 0.;
      RTKB_CUDA_TRY(cudaMemcpyAsync(&rr, c->scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st));
      RTKB_CUDA_TRY(cudaStreamSynchronize(st));
      if (rr < c->rr_best)
      {
        c->rr_best = rr;
        c->stall = 0;
      }
      else if (++c->stall >= kPcgPatience)
      {
        c->pcg_active = false;
        c->fallback_iteration = c->iterations;
        mul_kernel<float><<<grid_for(c->nvox), 256, 0, st>>>(c->P, c->R, nullptr, c->nvox); // restart: p = r
        RTKB_CUDA_TRY(cudaGetLastError());
      }
      continue;
    }
    cudaError_t e = c->exec ? cudaGraphLaunch(c->exec, st) : enqueue_iteration(c, st);
    if (e != cudaSuccess)
      return cuda_fail(e, "CG iteration");
    c->iterations++;
  }
  return RTKB_OK;
}

extern "C" int
rtkb_cg_residual(rtkb_cg * c, double * rr, double * rr0, int * iterations, void * stream)
{
  using namespace rtkb;
  if (!c)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null plan");
  double       h[2] = { 0., 0. };
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RTKB_CUDA_TRY(cudaMemcpyAsync(h, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  RTKB_CUDA_TRY(cudaStreamSynchronize(st));
  if (rr)
    *rr = h[S_RR];
  if (rr0)
    *rr0 = h[S_RR0];
  if (iterations)
    *iterations = c->iterations;
  return RTKB_OK;
}

// ---- checkpoint of a CG plan between iterations --------------------------------------------------
// Layout: a 64-byte header (magic, version, voxels, storage, iterations), the five FP64 scalars
// (rr, rr0, alpha, beta, pAp), R and P in the plan's storage types.
namespace
{
constexpr unsigned long long kStateMagic = 0x3174617453474342ull; // "BCGStat1" in little-endian bytes
struct StateHeader
{
  unsigned long long magic;
  long long          nvox;
  int                version, storage, iterations, pad;
  char               reserved[32];
};
static_assert(sizeof(StateHeader) == 64, "state header size");

int
plan_storage(const rtkb_cg * c)
{
  return c->bf16 ? 1 : (c->bf16p ? 2 : 0);
}

size_t
r_bytes(const rtkb_cg * c)
{
  return (size_t)c->nvox * (c->bf16 ? 2 : 4);
}

size_t
p_bytes(const rtkb_cg * c)
{
  return (size_t)c->nvox * ((c->bf16 || c->bf16p) ? 2 : 4);
}

int
state_check(const rtkb_cg * c)
{
  if (!c)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null plan");
  if (c->net)
    return rtkb::fail(RTKB_ERR_UNSUPPORTED, "the state of a plan with a learned preconditioner is not saved");
  return RTKB_OK;
}
} // namespace

extern "C" int
rtkb_cg_state_bytes(const rtkb_cg * c, long long * bytes)
{
  int rc = state_check(c);
  if (rc != RTKB_OK)
    return rc;
  if (!bytes)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = (long long)(sizeof(StateHeader) + 5 * sizeof(double) + r_bytes(c) + p_bytes(c));
  return RTKB_OK;
}

extern "C" int
rtkb_cg_save_state(rtkb_cg * c, void * buffer, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  int rc = state_check(c);
  if (rc != RTKB_OK)
    return rc;
  if (!buffer)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  StateHeader  h{};
  h.magic = kStateMagic;
  h.nvox = c->nvox;
  h.version = 1;
  h.storage = plan_storage(c);
  h.iterations = c->iterations;
  char * b = static_cast<char *>(buffer);
  RTKB_CUDA_TRY(cudaMemcpyAsync(b + sizeof(h), c->scal, 5 * sizeof(double), cudaMemcpyDefault, st));
  RTKB_CUDA_TRY(cudaMemcpyAsync(b + sizeof(h) + 5 * sizeof(double), c->R, r_bytes(c), cudaMemcpyDefault, st));
  RTKB_CUDA_TRY(
    cudaMemcpyAsync(b + sizeof(h) + 5 * sizeof(double) + r_bytes(c), c->P, p_bytes(c), cudaMemcpyDefault, st));
  // the header last, from this frame: synchronous with respect to the host for pageable memory, so
  // wait for the stream before h goes out of scope
  RTKB_CUDA_TRY(cudaMemcpyAsync(b, &h, sizeof(h), cudaMemcpyDefault, st));
  RTKB_CUDA_TRY(cudaStreamSynchronize(st));
  return RTKB_OK;
}

extern "C" int
rtkb_cg_load_state(rtkb_cg * c, const void * buffer, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  int rc = state_check(c);
  if (rc != RTKB_OK)
    return rc;
  if (!buffer)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  if (!c->x)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "start the plan (rtkb_cg_start) with the saved iterate first");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  StateHeader  h{};
  RTKB_CUDA_TRY(cudaStreamSynchronize(st));
  RTKB_CUDA_TRY(cudaMemcpy(&h, buffer, sizeof(h), cudaMemcpyDefault));
  if (h.magic != kStateMagic || h.version != 1)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "not a CG state");
  if (h.nvox != c->nvox || h.storage != plan_storage(c) || h.iterations < 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "the state belongs to a plan of another size or storage");
  const char * b = static_cast<const char *>(buffer);
  RTKB_CUDA_TRY(cudaMemcpyAsync(c->scal, b + sizeof(h), 5 * sizeof(double), cudaMemcpyDefault, st));
  RTKB_CUDA_TRY(cudaMemcpyAsync(c->R, b + sizeof(h) + 5 * sizeof(double), r_bytes(c), cudaMemcpyDefault, st));
  RTKB_CUDA_TRY(
    cudaMemcpyAsync(c->P, b + sizeof(h) + 5 * sizeof(double) + r_bytes(c), p_bytes(c), cudaMemcpyDefault, st));
  c->iterations = h.iterations;
  return RTKB_OK;
}

extern "C" void
rtkb_cg_destroy(rtkb_cg * c)
{
  release(c);
}

extern "C" int
rtkb_cg_set_support_mask(rtkb_cg * c, const float * d_mask)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null plan");
  if (d_mask && (c->bf16 || c->bf16p))
    return fail(RTKB_ERR_UNSUPPORTED, "support masks need an FP32 plan");
  if (d_mask && c->net)
    return fail(RTKB_ERR_UNSUPPORTED, "support masks and the learned preconditioner do not combine");
  if (d_mask && !c->Mx)
    RTKB_CUDA_TRY(cudaMalloc(&c->Mx, (size_t)c->nvox * 4));
  c->mask = d_mask;
  drop_graphs(c); // the next start captures the masked operator
  c->x = nullptr; // a run must start again
  return RTKB_OK;
}

extern "C" int
rtkb_cg_finish(rtkb_cg * c, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c || !c->x)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "CG plan not started");
  if (!c->mask)
    return RTKB_OK;
  mask_inplace_kernel<<<grid_for(c->nvox), 256, 0, static_cast<cudaStream_t>(stream)>>>(c->x, c->mask, c->nvox);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "CG support mask");
}

extern "C" int
rtkb_conjugate_gradient(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                        const rtkb_cg_params * params, const float * d_proj, const float * d_weights,
                        int displaced_detector, float * d_x, int max_iterations, double relative_residual,
                        int * iterations, double * final_relative_residual, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  rtkb_cg * c = nullptr;
  int       rc = rtkb_cg_create(g, vol, proj, params, &c);
  if (rc != RTKB_OK)
    return rc;
  rc = rtkb_cg_start(c, d_proj, d_weights, displaced_detector, d_x, stream);
  double rr = 0., rr0 = 0.;
  int    it = 0;
  for (; rc == RTKB_OK && it < max_iterations; it++)
  {
    if (relative_residual > 0.)
    {
      rc = rtkb_cg_residual(c, &rr, &rr0, nullptr, stream);
      if (rc != RTKB_OK || rr <= relative_residual * relative_residual * rr0)
        break;
    }
    rc = rtkb_cg_iterate(c, 1, stream);
  }
  if (rc == RTKB_OK)
    rc = rtkb_cg_residual(c, &rr, &rr0, nullptr, stream);
  if (iterations)
    *iterations = it;
  if (final_relative_residual)
    *final_relative_residual = rr0 > 0. ? std::sqrt(rr / rr0) : 0.;
  rtkb_cg_destroy(c);
  return rc;
}

extern "C" int
rtkb_cg_set_preconditioner(rtkb_cg * c, rtkb_unet * net, int history)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null plan");
  if (net && (history < 1 || history > kMaxHistory))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "history must be in 1..16");
  if (net && (c->bf16 || c->bf16p))
    return fail(RTKB_ERR_UNSUPPORTED, "the learned preconditioner runs on FP32 plans only");
  drop_graphs(c);
  c->x = nullptr; // must be started again
  c->net = nullptr;
  c->pcg_active = false;
  if (!net)
    return RTKB_OK;
  const int nx = c->vol.size[0], ny = c->vol.size[1], nz = c->vol.size[2];
  int       rc = rtkb_unet_reserve(net, 1, nx, ny, nz);
  if (rc != RTKB_OK)
    return rc;
  if (c->pmem && c->m != history)
  {
    cudaFree(c->pmem);
    c->pmem = nullptr;
  }
  if (!c->pmem)
  {
    const size_t vb = ((size_t)c->nvox * 4 + 255) & ~size_t(255);
    const size_t rb = kRedBlocks * sizeof(double);
    const size_t total = vb * (1 + 2 * (size_t)history) + rb * (1 + history) + (2 * history + 1) * sizeof(double);
    RTKB_CUDA_TRY(cudaMalloc(&c->pmem, total));
    char * m = static_cast<char *>(c->pmem);
    c->Z = reinterpret_cast<float *>(m);
    m += vb;
    c->Ph = reinterpret_cast<float *>(m);
    m += vb * history;
    c->APh = reinterpret_cast<float *>(m);
    m += vb * history;
    c->partial2 = reinterpret_cast<double *>(m);
    m += rb;
    c->mpartial = reinterpret_cast<double *>(m);
    m += rb * history;
    c->hist = reinterpret_cast<double *>(m);
    c->m = history;
    // zero so that never-written slots contribute nothing (beta_j = 0, 0 * p_j)
    RTKB_CUDA_TRY(cudaMemset(c->Ph, 0, 2 * vb * history));
  }
  c->net = net;
  return RTKB_OK;
}

extern "C" int
rtkb_cg_preconditioner_status(const rtkb_cg * c, int * active, int * fallback_iteration)
{
  using namespace rtkb;
  if (!c)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null plan");
  if (active)
    *active = c->pcg_active ? 1 : 0;
  if (fallback_iteration)
    *fallback_iteration = c->fallback_iteration;
  return RTKB_OK;
}

extern "C" int
rtkb_cg_apply_operator(rtkb_cg * c, const float * d_in, float * d_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!c || !d_in || !d_out || d_in == d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null or aliased argument");
  const cudaError_t e = apply_A(c, d_in, Elem::F32, d_out, Elem::F32, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "normal operator");
}

// ---------------------------------------------------------------- batched CG
// Many independent CG problems (the batched configuration's 10-iteration CG
// half): one plan per problem, eager (no per-plan graph), and ONE CUDA graph
// holding every problem's iterations, each problem's chain on its own forked
// capture stream.  A replay is a single launch; the problems' kernels run
// concurrently wherever their grids leave the GPU room.
struct rtkb_cg_batch
{
  std::vector<rtkb_cg *>    plans;
  std::vector<cudaStream_t> streams; // capture branches
  std::vector<cudaEvent_t>  joins;
  cudaEvent_t               fork = nullptr;
  cudaStream_t              cap = nullptr;
  cudaGraph_t               graph = nullptr;
  cudaGraphExec_t           exec = nullptr;
  int                       graph_iterations = 0; // iterations per problem in the captured graph
  bool                      started = false;
};

namespace
{
void
drop_batch_graph(rtkb_cg_batch * b)
{
  if (b->exec)
    cudaGraphExecDestroy(b->exec);
  if (b->graph)
    cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_iterations = 0;
}

void
release_batch(rtkb_cg_batch * b)
{
  if (!b)
    return;
  drop_batch_graph(b);
  for (rtkb_cg * c : b->plans)
    release(c);
  for (cudaStream_t s : b->streams)
    cudaStreamDestroy(s);
  for (cudaEvent_t e : b->joins)
    cudaEventDestroy(e);
  if (b->fork)
    cudaEventDestroy(b->fork);
  if (b->cap)
    cudaStreamDestroy(b->cap);
  delete b;
}

// capture niter iterations of every plan: fork from the capture stream, one
// branch per plan, join back
cudaError_t
capture_batch(rtkb_cg_batch * b, int niter)
{
  cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return e;
  cudaError_t ei = cudaEventRecord(b->fork, b->cap);
  for (size_t i = 0; i < b->plans.size() && ei == cudaSuccess; i++)
  {
    ei = cudaStreamWaitEvent(b->streams[i], b->fork, 0);
    for (int k = 0; k < niter && ei == cudaSuccess; k++)
      ei = enqueue_iteration(b->plans[i], b->streams[i]);
    if (ei == cudaSuccess)
      ei = cudaEventRecord(b->joins[i], b->streams[i]);
    if (ei == cudaSuccess)
      ei = cudaStreamWaitEvent(b->cap, b->joins[i], 0);
  }
  e = cudaStreamEndCapture(b->cap, &b->graph);
  if (e == cudaSuccess)
    e = ei;
  if (e == cudaSuccess)
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e == cudaSuccess)
    b->graph_iterations = niter;
  return e;
}
} // namespace

extern "C" int
rtkb_cg_batch_create(const rtkb_cg_batch_problem * problems, int n, const rtkb_cg_params * params,
                     rtkb_cg_batch ** out)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!out || !problems || n <= 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument or empty batch");
  *out = nullptr;
  rtkb_cg_params p = params ? *params : rtkb_cg_params{ 0., 1, 0 };
  p.use_cuda_graph = 0; // the batch captures all plans in one graph
  rtkb_cg_batch * b = nullptr;
  try
  {
    b = new rtkb_cg_batch();
    for (int i = 0; i < n; i++)
    {
      const rtkb_cg_batch_problem & q = problems[i];
      if (!q.d_proj || !q.d_x)
      {
        release_batch(b);
        return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer in batch problem");
      }
      rtkb_cg * c = nullptr;
      const int rc = rtkb_cg_create(q.geometry, &q.vol, &q.proj, &p, &c);
      if (rc != RTKB_OK)
      {
        release_batch(b);
        return rc;
      }
      b->plans.push_back(c);
      cudaStream_t s = nullptr;
      cudaEvent_t  ev = nullptr;
      cudaError_t  e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
      if (e == cudaSuccess)
        b->streams.push_back(s);
      if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess)
        b->joins.push_back(ev);
      if (e != cudaSuccess)
      {
        release_batch(b);
        return cuda_fail(e, "batch streams");
      }
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e != cudaSuccess)
    {
      release_batch(b);
      return cuda_fail(e, "batch streams");
    }
  }
  catch (...)
  {
    release_batch(b);
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  *out = b;
  return RTKB_OK;
}

extern "C" int
rtkb_cg_batch_start(rtkb_cg_batch * b, const rtkb_cg_batch_problem * problems, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!b || !problems)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  drop_batch_graph(b);
  for (size_t i = 0; i < b->plans.size(); i++)
  {
    const rtkb_cg_batch_problem & q = problems[i];
    const int rc = rtkb_cg_start(b->plans[i], q.d_proj, q.d_weights, q.displaced_detector, q.d_x, stream);
    if (rc != RTKB_OK)
      return rc;
  }
  b->started = true;
  return RTKB_OK;
}

extern "C" int
rtkb_cg_batch_iterate(rtkb_cg_batch * b, int niter, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!b || !b->started || niter < 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "batch not started");
  if (niter == 0)
    return RTKB_OK;
  if (b->graph_iterations != niter)
  {
    drop_batch_graph(b);
    const cudaError_t e = capture_batch(b, niter);
    if (e != cudaSuccess)
    {
      drop_batch_graph(b);
      return cuda_fail(e, "batched CG graph capture");
    }
  }
  RTKB_CUDA_TRY(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
  for (rtkb_cg * c : b->plans)
    c->iterations += niter;
  return RTKB_OK;
}

extern "C" rtkb_cg *
rtkb_cg_batch_plan(rtkb_cg_batch * b, int i)
{
  if (!b || i < 0 || i >= (int)b->plans.size())
    return nullptr;
  return b->plans[i];
}

extern "C" void
rtkb_cg_batch_destroy(rtkb_cg_batch * b)
{
  release_batch(b);
}

extern "C" int
rtkb_laplacian(const rtkb_image_desc * vol, const float * d_in, float * d_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!vol || !d_in || !d_out || d_in == d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null or aliased argument");
  if (!desc_valid(vol, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const cudaError_t e = laplacian_launch(*vol, d_in, d_out, 1.f, false, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "laplacian");
}
