// Smoothed isotropic total variation of a 2-D image and its gradient, the
// regulariser of the sparse-view model-based reconstruction that drives the
// differentiable back-projection (no counterpart in the reference, which
// has no iterative reconstruction on this path):
//     TV(x) = sum_{i < ny-1, j < nx-1} t_ij,
//     t_ij  = sqrt(dx_ij^2 + dy_ij^2 + eps),
//     dx_ij = x[i][j+1] - x[i][j],  dy_ij = x[i+1][j] - x[i][j].
// As tensor operations that is about ten launches each way over the image;
// here it is one launch for the value (plus a fixed-order reduction of the
// block partials) and one for the gradient
//     dTV/dx[i][j] = -(dx_ij + dy_ij) / t_ij        (i < ny-1, j < nx-1)
//                  + dx_{i,j-1} / t_{i,j-1}          (i < ny-1, j >= 1)
//                  + dy_{i-1,j} / t_{i-1,j}          (i >= 1, j < nx-1),
// scaled by an upstream gradient read from device memory (no host sync).
// Differences and t in FP32 (as the tensor form computes them); the value
// sums the t_ij in FP64 in a fixed order.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kValueBlocks = 592;  // 4 per SM: partials of the value

__device__ __forceinline__ float t_at(const float *x, long long rs, int i, int j, float eps, float &dx, float &dy) {
  const float c = __ldg(x + i * rs + j);
  dx = __ldg(x + i * rs + j + 1) - c;
  dy = __ldg(x + (i + 1) * rs + j) - c;
  return sqrtf(fmaf(dx, dx, fmaf(dy, dy, eps)));
}

__global__ void __launch_bounds__(kThreads) tv_value_kernel(const float *__restrict__ x, long long rs, int ny, int nx,
                                                            float eps, double *partial) {
  __shared__ double red[kThreads / 32];
  const long long nt = (long long)(ny - 1) * (nx - 1);
  double acc = 0.0;
  for (long long e = blockIdx.x * (long long)kThreads + threadIdx.x; e < nt; e += (long long)gridDim.x * kThreads) {
    const int i = (int)(e / (nx - 1)), j = (int)(e - (long long)i * (nx - 1));
    float dx, dy;
    acc += (double)t_at(x, rs, i, j, eps, dx, dy);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) s += red[k];
    partial[blockIdx.x] = s;
  }
}

// the block partials in a fixed order
__global__ void __launch_bounds__(32) tv_sum_kernel(const double *partial, int n, float *out) {
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += 32) acc += partial[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0) *out = (float)acc;
}

__global__ void __launch_bounds__(kThreads) tv_grad_kernel(const float *__restrict__ x, long long rs, int ny, int nx,
                                                           float eps, const float *__restrict__ scale, float weight,
                                                           float *g, long long grs, int accumulate) {
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i = blockIdx.y * (kThreads / 32) + (threadIdx.x >> 5);
  if (i >= ny || j >= nx) return;
  float v = 0.f, dx, dy;
  if (i < ny - 1 && j < nx - 1) {
    const float t = t_at(x, rs, i, j, eps, dx, dy);
    v -= (dx + dy) / t;
  }
  if (i < ny - 1 && j >= 1) {
    const float t = t_at(x, rs, i, j - 1, eps, dx, dy);
    v += dx / t;
  }
  if (i >= 1 && j < nx - 1) {
    const float t = t_at(x, rs, i - 1, j, eps, dx, dy);
    v += dy / t;
  }
  const float s = weight * (scale ? __ldg(scale) : 1.f);
  float *o = g + i * grs + j;
  *o = accumulate ? fmaf(s, v, *o) : s * v;
}

}  // namespace

extern "C" int64_t atb_tv_workspace(void) { return (int64_t)kValueBlocks * (int64_t)sizeof(double); }

extern "C" int atb_tv_value(const float *img, int64_t row_stride, int ny, int nx, double eps, void *workspace,
                            int64_t workspace_bytes, float *out, void *stream) {
  if (!img || !out || !workspace) return atb::fail(ATB_EINVAL, "atb_tv_value: null pointer");
  if (ny < 1 || nx < 1 || row_stride < nx) return atb::fail(ATB_EINVAL, "atb_tv_value: bad shape %dx%d", ny, nx);
  if (workspace_bytes < atb_tv_workspace())
    return atb::fail(ATB_EINVAL, "atb_tv_value: workspace of %lld bytes needed", (long long)atb_tv_workspace());
  cudaStream_t st = atb::as_stream(stream);
  double *part = static_cast<double *>(workspace);
  const long long nt = (long long)(ny - 1) * (nx - 1);
  int blocks = (int)std::min<long long>(kValueBlocks, std::max<long long>(1, (nt + kThreads - 1) / kThreads));
  tv_value_kernel<<<blocks, kThreads, 0, st>>>(img, row_stride, ny, nx, (float)eps, part);
  int rc = atb::check_launch("atb_tv_value");
  if (rc != ATB_OK) return rc;
  tv_sum_kernel<<<1, 32, 0, st>>>(part, blocks, out);
  return atb::check_launch("atb_tv_value (sum)");
}

extern "C" int atb_tv_grad(const float *img, int64_t row_stride, int ny, int nx, double eps, const float *scale,
                           float weight, float *grad, int64_t grad_row_stride, int accumulate, void *stream) {
  if (!img || !grad) return atb::fail(ATB_EINVAL, "atb_tv_grad: null pointer");
  if (ny < 1 || nx < 1 || row_stride < nx || grad_row_stride < nx)
    return atb::fail(ATB_EINVAL, "atb_tv_grad: bad shape %dx%d", ny, nx);
  if ((ny + kThreads / 32 - 1) / (kThreads / 32) > 65535)
    return atb::fail(ATB_ERANGE, "atb_tv_grad: %d rows too many", ny);
  const dim3 grid((nx + 31) / 32, (ny + kThreads / 32 - 1) / (kThreads / 32));
  tv_grad_kernel<<<grid, kThreads, 0, atb::as_stream(stream)>>>(img, row_stride, ny, nx, (float)eps, scale, weight,
                                                                 grad, grad_row_stride, accumulate ? 1 : 0);
  return atb::check_launch("atb_tv_grad");
}
