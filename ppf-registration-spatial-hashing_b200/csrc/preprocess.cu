// Driver-side preprocessing of the reference's alignment program on the GPU
// (src/alignment.cpp:203-288): the axis-aligned extent of a cloud (its
// model_d_dist = tau_d * largest extent, pcl::getMinMax3D) and voxel-grid
// downsampling (pcl::VoxelGrid<pcl::PointNormal> with one leaf size,
// src/alignment.cpp:79-87).
//
// VoxelGrid is PCL 1.8 code, absent here; its published algorithm is:
// inverse leaf size 1/leaf (float); min_b = floor(min * inv), max_b =
// floor(max * inv) over the cloud's extent; each point's cell offsets
// (int)(floor(p * inv) - (float)min_b) per axis, linear index i + j * dx +
// k * dx * dy with d = max_b - min_b + 1; points sorted by that index; every
// non-empty voxel, in index order, becomes the float mean of its points' x,
// y, z and normal components (normals are averaged, not renormalised).  When
// the grid would exceed 2^31 - 1 cells the input is returned unchanged.  Here
// the sort is stable, so each voxel sums its points in input order, with
// correctly rounded adds and divisions.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <climits>

#include "engine.h"

namespace ppf {
namespace {

// Ordered-integer image of a float (monotone for all non-NaN values), so
// min/max reduce with integer atomics.
__device__ __forceinline__ int ordered(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ __forceinline__ float unordered(int i) {
#ifdef __CUDA_ARCH__
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
#else
  const int j = i >= 0 ? i : i ^ 0x7fffffff;
  float f;
  std::memcpy(&f, &j, 4);
  return f;
#endif
}

// ext[0..2] = ordered min, ext[3..5] = ordered max over finite points.
__global__ void extent_kernel(const float* __restrict__ xyz, size_t n, int* __restrict__ ext) {
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
    const int o[3] = {ordered(x), ordered(y), ordered(z)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = min(lo[k], o[k]);
      hi[k] = max(hi[k], o[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    for (int off = 16; off; off >>= 1) {
      lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
      hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(ext + k, lo[k]);
      atomicMax(ext + 3 + k, hi[k]);
    }
  }
}

struct Grid {
  float inv;         // 1 / leaf
  int min_b[3];
  int div_x, div_xy;  // linear index multipliers
};

// Linear voxel index of each point (0xffffffff for a non-finite point).
__global__ void voxel_index_kernel(const float* __restrict__ xyz, size_t n, Grid g, uint32_t* __restrict__ idx) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
      idx[i] = 0xffffffffu;
      continue;
    }
    const int i0 = (int)__fsub_rn(floorf(__fmul_rn(x, g.inv)), (float)g.min_b[0]);
    const int i1 = (int)__fsub_rn(floorf(__fmul_rn(y, g.inv)), (float)g.min_b[1]);
    const int i2 = (int)__fsub_rn(floorf(__fmul_rn(z, g.inv)), (float)g.min_b[2]);
    idx[i] = (uint32_t)(i0 + i1 * g.div_x + i2 * g.div_xy);
  }
}

// Mean of each voxel's points (stable order), written in voxel order.
__global__ void centroid_kernel(const uint32_t* __restrict__ first, const uint32_t* __restrict__ count,
                                size_t K, const uint32_t* __restrict__ order, const float* __restrict__ xyz,
                                const float* __restrict__ nxyz, float* __restrict__ out_xyz,
                                float* __restrict__ out_nxyz) {
  for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < K; v += (size_t)gridDim.x * blockDim.x) {
    float s[6] = {0, 0, 0, 0, 0, 0};
    const uint32_t f = first[v], c = count[v];
    for (uint32_t k = 0; k < c; ++k) {
      const size_t p = order[f + k];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s[d] = __fadd_rn(s[d], xyz[3 * p + d]);
        s[3 + d] = __fadd_rn(s[3 + d], nxyz[3 * p + d]);
      }
    }
    const float cf = (float)c;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      out_xyz[3 * v + d] = __fdiv_rn(s[d], cf);
      out_nxyz[3 * v + d] = __fdiv_rn(s[3 + d], cf);
    }
  }
}

__global__ void count_finite_kernel(const uint32_t* __restrict__ sorted_idx, size_t n, uint32_t* __restrict__ n_fin) {
  // sorted ascending: non-finite points (0xffffffff) come last
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (sorted_idx[i] != 0xffffffffu && (i + 1 == n || sorted_idx[i + 1] == 0xffffffffu)) *n_fin = (uint32_t)(i + 1);
}

}  // namespace

bool cloud_extent(Context& ctx, const float* xyz_dev, size_t n, float lo[3], float hi[3]) {
  DevBuf e;
  e.reserve(6 * sizeof(int));
  const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  PPF_CUDA(cudaMemcpyAsync(e.ptr, init, sizeof(init), cudaMemcpyHostToDevice, ctx.stream));
  if (n) {
    extent_kernel<<<grid_for(n, 256, 4), 256, 0, ctx.stream>>>(xyz_dev, n, e.as<int>());
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
  }
  int h[6];
  PPF_CUDA(cudaMemcpyAsync(h, e.ptr, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
  PPF_CUDA(cudaStreamSynchronize(ctx.stream));
  if (h[0] == INT_MAX) return false;  // no finite point
  for (int k = 0; k < 3; ++k) {
    lo[k] = unordered(h[k]);
    hi[k] = unordered(h[3 + k]);
  }
  return true;
}

size_t voxel_downsample(Context& ctx, const float* xyz_dev, const float* nxyz_dev, size_t n, float leaf,
                        DevBuf& out_xyz, DevBuf& out_nxyz) {
  cudaStream_t st = ctx.stream;
  PPF_REQUIRE(leaf > 0.f && std::isfinite(leaf), PPF_ERR_INVALID_ARGUMENT, "leaf size must be positive");
  PPF_REQUIRE(n < 0xffffffffull, PPF_ERR_INVALID_ARGUMENT, "cloud larger than 2^32 - 1 points");
  float lo[3], hi[3];
  auto copy_input = [&](size_t m) {
    out_xyz.reserve(std::max<size_t>(m, 1) * 12);
    out_nxyz.reserve(std::max<size_t>(m, 1) * 12);
    if (m) {
      PPF_CUDA(cudaMemcpyAsync(out_xyz.ptr, xyz_dev, m * 12, cudaMemcpyDeviceToDevice, st));
      PPF_CUDA(cudaMemcpyAsync(out_nxyz.ptr, nxyz_dev, m * 12, cudaMemcpyDeviceToDevice, st));
    }
    return m;
  };
  if (!cloud_extent(ctx, xyz_dev, n, lo, hi)) return 0;
  Grid g;
  g.inv = 1.0f / leaf;  // host float division, as Eigen's Ones() / leaf
  long long d[3];
  for (int k = 0; k < 3; ++k) d[k] = (long long)((hi[k] - lo[k]) * g.inv) + 1;
  // PCL 1.8 returns the input unchanged when the grid would overflow its int index
  if (d[0] * d[1] * d[2] > (long long)INT_MAX) return copy_input(n);
  int max_b[3];
  for (int k = 0; k < 3; ++k) {
    g.min_b[k] = (int)std::floor(lo[k] * g.inv);
    max_b[k] = (int)std::floor(hi[k] * g.inv);
  }
  const long long dx = max_b[0] - g.min_b[0] + 1, dy = max_b[1] - g.min_b[1] + 1,
                  dz = max_b[2] - g.min_b[2] + 1;
  PPF_REQUIRE(dx * dy * dz <= (long long)INT_MAX, PPF_ERR_INVALID_ARGUMENT, "voxel grid beyond 2^31 cells");
  g.div_x = (int)dx;
  g.div_xy = (int)(dx * dy);
  DevBuf idx, order, uniq, first, count;
  idx.reserve(n * 4);
  order.reserve(n * 4);
  voxel_index_kernel<<<grid_for(n, 256), 256, 0, st>>>(xyz_dev, n, g, idx.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 4, st));
  const size_t l0 = ctx.sort32.launches();
  ctx.sort32.sort(idx.as<uint32_t>(), order.as<uint32_t>(), true, n, 0, 32, st, ctx.flags.as<uint32_t>());
  ctx.launches += ctx.sort32.launches() - l0;
  // finite points only (their indices sort first)
  PPF_CUDA(cudaMemsetAsync(ctx.counters.ptr, 0, 4, st));
  count_finite_kernel<<<grid_for(n, 256), 256, 0, st>>>(idx.as<uint32_t>(), n, ctx.counters.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());
  uint32_t n_fin = 0;
  PPF_CUDA(cudaMemcpyAsync(&n_fin, ctx.counters.ptr, 4, cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  ctx.launches++;
  uniq.reserve(std::max<size_t>(n_fin, 1) * 4);
  first.reserve(std::max<size_t>(n_fin, 1) * 4);
  count.reserve(std::max<size_t>(n_fin, 1) * 4);
  const size_t K = n_fin ? build_runs(idx.as<uint32_t>(), n_fin, uniq.as<uint32_t>(), first.as<uint32_t>(),
                                      count.as<uint32_t>(), ctx.scratch, st, &ctx.launches)
                         : 0;
  out_xyz.reserve(std::max<size_t>(K, 1) * 12);
  out_nxyz.reserve(std::max<size_t>(K, 1) * 12);
  if (K) {
    centroid_kernel<<<grid_for(K, 128), 128, 0, st>>>(first.as<uint32_t>(), count.as<uint32_t>(), K,
                                                       order.as<uint32_t>(), xyz_dev, nxyz_dev,
                                                       out_xyz.as<float>(), out_nxyz.as<float>());
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
  }
  uint32_t flags = 0;
  PPF_CUDA(cudaMemcpyAsync(&flags, ctx.flags.ptr, 4, cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  PPF_REQUIRE(!(flags & kFlagSpinTimeout), PPF_ERR_TIMEOUT, "radix sort look-back timed out");
  return K;
}

}  // namespace ppf
