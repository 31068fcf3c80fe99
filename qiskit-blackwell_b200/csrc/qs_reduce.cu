// qs_reduce.cu — reductions over a state, accumulated in FP64 in a fixed
// order (no floating-point atomics), so every result is bit-reproducible and
// the same whether a state is processed alone or inside a batch.
//
// Two-stage scheme: stage 1 gives each block a fixed contiguous slice of the
// index range (the slicing depends only on the item count); every thread sums
// a fixed strided subset sequentially, then the block reduces in a fixed tree
// order.  Stage 2 is one block that reduces the per-block partials in order.
#include "qs_api.h"
#include <vector>
#include "qs_common.cuh"
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

using namespace qs;

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1024;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block reduction; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = 0.0;
  if (w == 0) {
    v = lane < nw ? ws[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

struct Slicing { int nb; uint64_t per; };
Slicing slice(uint64_t items) {
  uint64_t nb = (items + 4095) / 4096;
  if (nb > kMaxBlocks) nb = kMaxBlocks;
  if (nb < 1) nb = 1;
  return Slicing{(int)nb, (items + nb - 1) / nb};
}

// -------------------------------------------------------------- functors -
// Each functor sees "items" = float4 vectors (two amplitudes).
struct FNorm {
  const float4* s;
  __device__ double operator()(uint64_t i) const {
    float4 v = s[i];
    return (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
  }
};

struct FP0 {  // probability of bit t = 0
  const float4* s;
  int t;
  __device__ double operator()(uint64_t i) const {
    float4 v = s[i];
    double a = (double)v.x * v.x + (double)v.y * v.y;
    double b = (double)v.z * v.z + (double)v.w * v.w;
    if (t == 0) return a;
    return ((2 * i) >> t) & 1 ? 0.0 : a + b;
  }
};

struct FZ {  // sum |a_i|^2 (-1)^popc(i & z)
  const float4* s;
  uint64_t z;
  __device__ double operator()(uint64_t i) const {
    float4 v = s[i];
    double a = (double)v.x * v.x + (double)v.y * v.y;
    double b = (double)v.z * v.z + (double)v.w * v.w;
    uint64_t i0 = 2 * i;
    double s0 = (__popcll(i0 & z) & 1) ? -a : a;
    double s1 = (__popcll((i0 + 1) & z) & 1) ? -b : b;
    return s0 + s1;
  }
};

template <class F>
__global__ void k_reduce(F f, uint64_t items, uint64_t per, double* __restrict__ partial) {
  pdl_begin();
  const uint64_t b0 = (uint64_t)blockIdx.x * per;
  const uint64_t e = min(b0 + per, items);
  double acc = 0.0;
  for (uint64_t i = b0 + threadIdx.x; i < e; i += blockDim.x) acc += f(i);
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// mode 0: out[0] = sum.  mode 1: out[0] = sum, out[1] = 1/sqrt(sum) (renorm).
__global__ void k_final(const double* __restrict__ partial, int nb, double* __restrict__ out, int mode) {
  pdl_begin();
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += partial[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) {
    out[0] = acc;
    if (mode == 1) out[1] = acc > 0.0 ? 1.0 / sqrt(acc) : 0.0;
  }
}

__global__ void k_scale(float4* __restrict__ s, uint64_t nvec, const double* __restrict__ scale) {
  pdl_begin();
  const float f = (float)scale[1];
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    float4 v = s[i];
    s[i] = make_float4(v.x * f, v.y * f, v.z * f, v.w * f);
  }
}

__global__ void k_probs(const float4* __restrict__ s, float2* __restrict__ p, uint64_t nvec) {
  pdl_begin();
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    float4 v = s[i];
    p[i] = make_float2(v.x * v.x + v.y * v.y, v.z * v.z + v.w * v.w);
  }
}

// Collapse after measuring qubit t: keep amplitudes with bit t == outcome,
// scaled by 1/sqrt(p_outcome); zero the others.  pr[0] = P(bit = 0).
__global__ void k_collapse(float4* __restrict__ s, uint64_t nvec, int t, double u, const double* __restrict__ pr,
                           int* __restrict__ outcome) {
  pdl_begin();
  const double p0 = pr[0];
  const int res = (u < p0) ? 0 : 1;
  const double p = res == 0 ? p0 : 1.0 - p0;
  const float f = p > 1e-30 ? (float)(1.0 / sqrt(p)) : 0.f;
  if (blockIdx.x == 0 && threadIdx.x == 0) *outcome = res;
  for (uint64_t i = gtid(); i < nvec; i += gstride()) {
    float4 v = s[i];
    const uint64_t i0 = 2 * i;
    const int b0 = (int)((i0 >> t) & 1), b1 = (int)(((i0 + 1) >> t) & 1);
    const float f0 = b0 == res ? f : 0.f, f1 = b1 == res ? f : 0.f;
    s[i] = make_float4(v.x * f0, v.y * f0, v.z * f1, v.w * f1);
  }
}

// ----------------------------------------------------------- sampling ----
// The CDF is built in chunks of kChunk amplitudes.  A chunk is split into 32
// contiguous segments of kSeg amplitudes, one per lane; a lane sums its
// segment sequentially in FP64 and the warp scans the 32 segment sums in a
// fixed shuffle order.  The same routine (seg_sum_staged) produces the chunk
// totals (pass 1) and the in-chunk search (pass 3), so both see identical
// values.
constexpr int kSeg = 64;
constexpr int kChunk = 32 * kSeg;

// |a|^2 in FP64, and a segment's running sum: the one expression and order
// that every pass uses, so the chunk totals and the in-chunk search agree bit
// for bit.
__device__ __forceinline__ void seg_add(double& acc, float2 a) { acc += (double)a.x * a.x + (double)a.y * a.y; }

// Lane `lane`'s segment sum of the chunk starting at `c0`: its amplitudes
// c0 + lane * kSeg + k, k = 0..kSeg-1, added by seg_add in order.  The chunk
// is read in coalesced 128-byte runs (a segment is 512 contiguous bytes per
// lane, so loading it lane by lane would touch 32 lines per warp access): the
// warp stages 16 amplitudes of every segment at a time in `buf` (32 rows of
// 17: the pad spreads a row walk over the banks) and each lane adds its row.
__device__ __forceinline__ void seg_stage_load(const float2* __restrict__ s, uint64_t c0, uint64_t n, int lane, int q,
                                               float4 (&r)[8]) {
  // lanes 8k..8k+7 cover one 128-byte run (16 amplitudes of one segment),
  // two amplitudes per lane.  16-byte loads when the state starts on a
  // 16-byte boundary and has an even length (every state of one or more
  // qubits): g is even, so the pair is then either inside it or past its end
  const bool v4 = ((reinterpret_cast<uintptr_t>(s) & 15) == 0) && !(n & 1);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint64_t g = c0 + (uint64_t)(4 * i + (lane >> 3)) * kSeg + 16 * q + 2 * (lane & 7);
    if (v4 && g < n) {
      r[i] = *reinterpret_cast<const float4*>(s + g);
    } else {
      const float2 lo = g < n ? s[g] : make_float2(0.f, 0.f);
      const float2 hi = g + 1 < n ? s[g + 1] : make_float2(0.f, 0.f);
      r[i] = make_float4(lo.x, lo.y, hi.x, hi.y);
    }
  }
}
__device__ __forceinline__ double seg_sum_staged(const float2* __restrict__ s, uint64_t c0, uint64_t n, int lane,
                                                 float2 (*buf)[17]) {
  double acc = 0.0;
  float4 r[8];
  seg_stage_load(s, c0, n, lane, 0, r);
#pragma unroll 1
  for (int q = 0; q < kSeg / 16; ++q) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int row = 4 * i + (lane >> 3), e = 2 * (lane & 7);
      buf[row][e] = make_float2(r[i].x, r[i].y);
      buf[row][e + 1] = make_float2(r[i].z, r[i].w);
    }
    __syncwarp();
    if (q + 1 < kSeg / 16) seg_stage_load(s, c0, n, lane, q + 1, r);  // in flight while this row is summed
    const uint64_t start = c0 + (uint64_t)lane * kSeg + 16 * q;
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (start + k < n) seg_add(acc, buf[lane][k]);
    __syncwarp();
  }
  return acc;
}

// inclusive warp scan in fixed order
__device__ __forceinline__ double warp_iscan(double v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// pass 1: one warp per chunk -> csum[c]
__global__ void k_chunk_sums(const float2* __restrict__ s, uint64_t n, uint64_t nchunks, double* __restrict__ csum) {
  pdl_begin();
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ float2 stage[kThreads / 32][32][17];
  for (uint64_t c = warp; c < nchunks; c += nwarps) {
    double v = seg_sum_staged(s, c * kChunk, n, lane, stage[threadIdx.x >> 5]);
    v = warp_iscan(v);
    if (lane == 31) csum[c] = v;
  }
}

// pass 2: exclusive scan of the chunk sums, one block, fixed order.
// cbase[c] = sum_{c' < c} csum[c'];  cbase[nchunks] = total.  The order
// depends only on nchunks and the block size (1024 threads in every launch).
// Each thread owns a contiguous run of `per` chunks; the block walks the runs
// kScanCols columns at a time through a shared tile (one row per thread), so
// csum is read and cbase written in coalesced 64-byte runs while every thread
// still adds its own run in order.  The next columns are fetched into
// registers while the current tile is summed.
constexpr int kScanThreads = 1024;
constexpr int kScanCols = 8;
constexpr size_t kScanSmem = sizeof(double) * kScanThreads * (kScanCols + 1);
using ScanTile = double (*)[kScanCols + 1];

// element m of this thread's share of a tile is row tid / kScanCols +
// m * (kScanThreads / kScanCols), column tid % kScanCols: chunk
// c0 + k0 + m * cstride, with c0 = (tid / kScanCols) * per + tid % kScanCols.
// A state of at most 34 qubits has at most 2^23 chunks: 32-bit indices.
struct ScanCols {
  uint32_t c0, cstride;
  int col;
};
__device__ __forceinline__ ScanCols scan_cols(uint64_t per) {
  const int col = threadIdx.x % kScanCols;
  return {(uint32_t)((threadIdx.x / kScanCols) * per + col), (uint32_t)((kScanThreads / kScanCols) * per), col};
}

__device__ __forceinline__ void scan_tile_fetch(const double* __restrict__ csum, uint64_t nchunks, uint64_t per,
                                                const ScanCols& sc, uint64_t k0, double (&r)[kScanCols]) {
  const bool in_run = k0 + sc.col < per;
#pragma unroll
  for (int m = 0; m < kScanCols; ++m) {
    const uint32_t c = sc.c0 + (uint32_t)k0 + m * sc.cstride;
    r[m] = (in_run && c < nchunks) ? csum[c] : 0.0;
  }
}

__device__ __forceinline__ void scan_tile_put(const double (&r)[kScanCols], ScanTile tile) {
#pragma unroll
  for (int m = 0; m < kScanCols; ++m) {
    const int i = threadIdx.x + kScanThreads * m;
    tile[i / kScanCols][i % kScanCols] = r[m];
  }
}

__device__ __forceinline__ void scan_tile_store(double* __restrict__ cbase, uint64_t nchunks, uint64_t per,
                                                const ScanCols& sc, uint64_t k0, ScanTile tile) {
  const bool in_run = k0 + sc.col < per;
#pragma unroll
  for (int m = 0; m < kScanCols; ++m) {
    const uint32_t c = sc.c0 + (uint32_t)k0 + m * sc.cstride;
    const int i = threadIdx.x + kScanThreads * m;
    if (in_run && c < nchunks) cbase[c] = tile[i / kScanCols][i % kScanCols];
  }
}

__device__ __forceinline__ void chunk_scan_block(const double* __restrict__ csum, uint64_t nchunks,
                                                 double* __restrict__ cbase, double* ws, double& carry, ScanTile tile) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint64_t per = (nchunks + kScanThreads - 1) / kScanThreads;
  const uint64_t b = (uint64_t)tid * per, e = min(b + per, nchunks);
  const ScanCols sc = scan_cols(per);
  double r[kScanCols];
  double local = 0.0;
  scan_tile_fetch(csum, nchunks, per, sc, 0, r);
  for (uint64_t k0 = 0; k0 < per; k0 += kScanCols) {
    scan_tile_put(r, tile);
    __syncthreads();
    if (k0 + kScanCols < per) scan_tile_fetch(csum, nchunks, per, sc, k0 + kScanCols, r);
#pragma unroll
    for (int j = 0; j < kScanCols; ++j)
      if (b + k0 + j < e) local += tile[tid][j];
    __syncthreads();
  }
  // block exclusive scan of `local`
  double inc = warp_iscan(local);
  double exc = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exc = 0.0;
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int nw = kScanThreads >> 5;
    double x = lane < nw ? ws[lane] : 0.0;
    double xi = warp_iscan(x);
    double xe = __shfl_up_sync(0xffffffffu, xi, 1);
    if (lane == 0) xe = 0.0;
    __syncwarp();
    if (lane < nw) ws[lane] = xe;  // exclusive warp offsets
    if (lane == nw - 1) carry = xi;
  }
  __syncthreads();
  double run = ws[w] + exc;
  scan_tile_fetch(csum, nchunks, per, sc, 0, r);
  for (uint64_t k0 = 0; k0 < per; k0 += kScanCols) {
    scan_tile_put(r, tile);
    __syncthreads();
    if (k0 + kScanCols < per) scan_tile_fetch(csum, nchunks, per, sc, k0 + kScanCols, r);
#pragma unroll
    for (int j = 0; j < kScanCols; ++j) {
      if (b + k0 + j < e) {
        const double v = tile[tid][j];
        tile[tid][j] = run;
        run += v;
      }
    }
    __syncthreads();
    scan_tile_store(cbase, nchunks, per, sc, k0, tile);
    __syncthreads();
  }
  if (tid == 0) cbase[nchunks] = carry;
}

__global__ void __launch_bounds__(kScanThreads, 1)
    k_chunk_scan(const double* __restrict__ csum, uint64_t nchunks, double* __restrict__ cbase) {
  pdl_begin();
  __shared__ double ws[32];
  __shared__ double carry;
  extern __shared__ double scan_smem[];
  chunk_scan_block(csum, nchunks, cbase, ws, carry, reinterpret_cast<ScanTile>(scan_smem));
}

// pass 3, one shot by one warp: u -> smallest i with cdf[i] >= u, clamped to
// n-1 (reference semantics: sample_sm120.cu:61-68).  Every lane returns it.
__device__ __forceinline__ int64_t sample_one(const float2* __restrict__ s, uint64_t n, uint64_t nchunks,
                                              const double* __restrict__ cbase, double x, float2 (*buf)[17]) {
  const int lane = threadIdx.x & 31;
  // smallest chunk c with cbase[c+1] >= x (nchunks if none): a 32-way search,
  // each lane probing one of 32 evenly spaced chunks per round.  cbase is
  // non-decreasing, so this finds the same chunk as a binary search.
  // Invariant: the answer is in [lo, hi], and cbase[hi+1] >= x if hi < nchunks.
  uint64_t lo = 0, hi = nchunks;
  while (lo < hi) {
    const uint64_t step = (hi - lo + 31) >> 5;
    const uint64_t p = lo + (uint64_t)lane * step;
    const unsigned m = __ballot_sync(0xffffffffu, p < hi && cbase[p + 1] >= x);
    if (m != 0) {
      const int j = __ffs(m) - 1;
      const uint64_t pj = lo + (uint64_t)j * step;
      lo = j ? pj - step + 1 : pj;
      hi = pj;
    } else {
      lo += (hi - 1 - lo) / step * step + 1;  // past the last probed chunk
    }
  }
  if (lo >= nchunks) return (int64_t)(n - 1);
  const uint64_t c = lo;
  double v = seg_sum_staged(s, c * kChunk, n, lane, buf);
  double inc = warp_iscan(v);
  const double base = cbase[c];
  const bool hit = base + inc >= x;
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if (m == 0) return (int64_t)min((c + 1) * (uint64_t)kChunk, n) - 1;
  const int L = __ffs(m) - 1;
  // lane L walks its segment
  int64_t r = 0;
  if (lane == L) {
    double run = base + (inc - v);
    const uint64_t st = c * kChunk + (uint64_t)L * kSeg;
    uint64_t i = st;
    r = -1;
    for (int q = 0; q < kSeg; ++q, ++i) {
      if (i >= n) break;
      float2 a = s[i];
      run += (double)a.x * a.x + (double)a.y * a.y;
      if (run >= x) { r = (int64_t)i; break; }
    }
    if (r < 0) r = (int64_t)min(st + kSeg, n) - 1;
  }
  return __shfl_sync(0xffffffffu, r, L);
}

__global__ void k_sample(const float2* __restrict__ s, uint64_t n, uint64_t nchunks, const double* __restrict__ cbase,
                         const double* __restrict__ u, int64_t nshots, int64_t* __restrict__ out) {
  pdl_begin();
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ float2 stage[kThreads / 32][32][17];
  for (uint64_t k = warp; k < (uint64_t)nshots; k += nwarps) {
    const int64_t result = sample_one(s, n, nchunks, cbase, u[k], stage[threadIdx.x >> 5]);
    if (lane == 0) out[k] = result;
  }
}

// ------------------------------------------------- batched sampling ------
// Many states of any widths in three launches.  Each state's CDF is built and
// searched exactly as qs_sample does it (same chunking, scan order and
// search), and shot k of state t uses value k of seeds[t]'s uniform stream,
// so the shots equal qs_sample's with those uniforms.
struct SampleDesc {
  uint64_t state_off;  // first amplitude of the state
  uint64_t n;          // amplitudes (2^width)
  uint64_t nchunks;
  uint64_t chunk_off;  // prefix sum of nchunks
  uint64_t shot_off;   // prefix sum of shots
  uint64_t seed;
};

// last descriptor whose field `off` is <= g (descriptors sorted by it)
template <uint64_t SampleDesc::*F>
__device__ __forceinline__ int find_desc(const SampleDesc* __restrict__ d, int ns, uint64_t g) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].*F <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_chunk_sums_b(const float2* __restrict__ base, const SampleDesc* __restrict__ d, int ns,
                               uint64_t total_chunks, double* __restrict__ csum) {
  pdl_begin();
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ float2 stage[kThreads / 32][32][17];
  for (uint64_t g = warp; g < total_chunks; g += nwarps) {
    const int t = find_desc<&SampleDesc::chunk_off>(d, ns, g);
    const SampleDesc D = d[t];
    const uint64_t c = g - D.chunk_off;
    double v = seg_sum_staged(base + D.state_off, c * kChunk, D.n, lane, stage[threadIdx.x >> 5]);
    v = warp_iscan(v);
    if (lane == 31) csum[g] = v;
  }
}

// one 1024-thread block per state; cbase of state t starts at chunk_off + t
__global__ void __launch_bounds__(kScanThreads, 1)
    k_chunk_scan_b(const double* __restrict__ csum, const SampleDesc* __restrict__ d, double* __restrict__ cbase) {
  pdl_begin();
  __shared__ double ws[32];
  __shared__ double carry;
  extern __shared__ double scan_smem[];
  const SampleDesc D = d[blockIdx.x];
  if (D.shot_off == d[blockIdx.x + 1].shot_off) return;  // no shots: nothing to scan (block-uniform)
  chunk_scan_block(csum + D.chunk_off, D.nchunks, cbase + D.chunk_off + blockIdx.x, ws, carry,
                   reinterpret_cast<ScanTile>(scan_smem));
}

__global__ void k_sample_b(const float2* __restrict__ base, const SampleDesc* __restrict__ d, int ns,
                           uint64_t total_shots, const double* __restrict__ cbase, int64_t* __restrict__ out) {
  pdl_begin();
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ float2 stage[kThreads / 32][32][17];
  for (uint64_t g = warp; g < total_shots; g += nwarps) {
    const int t = find_desc<&SampleDesc::shot_off>(d, ns, g);
    const SampleDesc D = d[t];
    const double x = qs_seed_uniform_at(D.seed, g - D.shot_off);
    const int64_t result =
        sample_one(base + D.state_off, D.n, D.nchunks, cbase + D.chunk_off + t, x, stage[threadIdx.x >> 5]);
    if (lane == 0) out[g] = result;
  }
}

// ---------------------------------------------------- Pauli-sum terms ----
// Term t: coefficient w_t = coef_t * i^{popc(x_t & z_t)} (complex), x_t, z_t.
// (P psi)[i] = i^{|x&z|} (-1)^{popc((i^x) & z)} psi[i ^ x].
struct Term { uint64_t x, z; double wr, wi; };

__device__ __forceinline__ void term_apply(const Term& T, uint64_t i, const float2* __restrict__ s, double& re,
                                           double& im) {
  const uint64_t j = i ^ T.x;
  const float2 b = s[j];
  const double sg = (__popcll(j & T.z) & 1) ? -1.0 : 1.0;
  re += sg * (T.wr * b.x - T.wi * b.y);
  im += sg * (T.wr * b.y + T.wi * b.x);
}

// <psi|H|psi> partials: sum_i Re(conj(psi_i) (H psi)_i)
__global__ void k_pauli_expect(const float2* __restrict__ s, uint64_t n, const Term* __restrict__ terms, int nterms,
                               uint64_t per, double* __restrict__ partial) {
  pdl_begin();
  extern __shared__ Term st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  const uint64_t b0 = (uint64_t)blockIdx.x * per;
  const uint64_t e = min(b0 + per, n);
  double acc = 0.0;
  for (uint64_t i = b0 + threadIdx.x; i < e; i += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nterms; ++k) term_apply(st[k], i, s, re, im);
    const float2 a = s[i];
    acc += (double)a.x * re + (double)a.y * im;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// out = H psi (complex64), accumulated in FP64 per amplitude.
__global__ void k_pauli_apply(const float2* __restrict__ s, float2* __restrict__ out, uint64_t n,
                              const Term* __restrict__ terms, int nterms) {
  pdl_begin();
  extern __shared__ Term st[];
  for (int k = threadIdx.x; k < nterms; k += blockDim.x) st[k] = terms[k];
  __syncthreads();
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nterms; ++k) term_apply(st[k], i, s, re, im);
    out[i] = make_float2((float)re, (float)im);
  }
}

}  // namespace

// Builds the device term table (records of {x, z, w_re, w_im}) in scratch
// after `offset` bytes.
void* qs_upload_terms(qs_context* h, size_t offset, int n, const uint64_t* x, const uint64_t* z, const double* c,
                      int nterms);

void* qs_upload_terms(qs_context* h, size_t offset, int n, const uint64_t* x, const uint64_t* z, const double* c,
                      int nterms) {
  QS_CHECK_ARG(nterms >= 1, "need at least one Pauli term");
  QS_CHECK_ARG(x && z && c, "term pointers are null");
  const uint64_t lim = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  std::vector<Term> T(nterms);
  for (int k = 0; k < nterms; ++k) {
    QS_CHECK_ARG((x[k] & ~lim) == 0 && (z[k] & ~lim) == 0, "Pauli mask has bits beyond n_qubits");
    const int ny = __builtin_popcountll(x[k] & z[k]) & 3;
    // i^ny
    static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, 1, 0, -1};
    T[k] = Term{x[k], z[k], c[k] * pr[ny], c[k] * pi[ny]};
  }
  char* base = (char*)h->scratch_get(offset + sizeof(Term) * nterms);
  Term* d = (Term*)(base + offset);
  // From pageable memory the copy returns once T has been staged, so the
  // host vector may go out of scope afterwards.
  QS_CUDA(cudaMemcpyAsync(d, T.data(), sizeof(Term) * nterms, cudaMemcpyHostToDevice, h->stream));
  return d;
}

namespace {

template <class F>
void reduce_to(qs_context* h, F f, uint64_t items, double* d_out, int mode, double* d_partial) {
  Slicing sl = slice(items);
  qs_launch_pdl(h, k_reduce<F>, dim3(sl.nb), dim3(kThreads), 0, f, items, sl.per, d_partial);
  qs_after_launch(h, "k_reduce");
  qs_launch_pdl(h, k_final, dim3(1), dim3(1024), 0, d_partial, sl.nb, d_out, mode);
  qs_after_launch(h, "k_final");
}

// scratch layout for reductions: [0, 16) two doubles out; [64, ...) partials
double* red_out(qs_context* h) { return (double*)h->scratch_get(64 + 8 * kMaxBlocks); }
double* red_part(qs_context* h) { return (double*)((char*)h->scratch_get(64 + 8 * kMaxBlocks) + 64); }

double fetch_scalar(qs_context* h, const double* d) {
  double* pin = h->pinned_get(64);
  QS_CUDA(cudaMemcpyAsync(pin, d, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  QS_CUDA(cudaStreamSynchronize(h->stream));
  return pin[0];
}

}  // namespace

extern "C" {

int qs_norm2(qs_handle_t h, const void* state, int n, double* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(out != nullptr, "out is null");
  double* o = red_out(h);
  reduce_to(h, FNorm{(const float4*)state}, (1ull << n) / 2, o, 0, red_part(h));
  *out = fetch_scalar(h, o);
  QS_API_END(h)
}

int qs_renorm(qs_handle_t h, void* state, int n) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  double* o = red_out(h);
  const uint64_t nvec = (1ull << n) / 2;
  reduce_to(h, FNorm{(const float4*)state}, nvec, o, 1, red_part(h));
  qs_launch_pdl(h, k_scale, dim3(qs_blocks_for(h, nvec, kThreads)), dim3(kThreads), 0, (float4*)state, nvec, o);
  qs_after_launch(h, "k_scale");
  QS_API_END(h)
}

int qs_probs(qs_handle_t h, const void* state, int n, float* probs) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(probs != nullptr && ((uintptr_t)probs & 7u) == 0, "probs must be a non-null 8-byte aligned pointer");
  const uint64_t nvec = (1ull << n) / 2;
  qs_launch_pdl(h, k_probs, dim3(qs_blocks_for(h, nvec, kThreads)), dim3(kThreads), 0, (const float4*)state, (float2*)probs, nvec);
  qs_after_launch(h, "k_probs");
  QS_API_END(h)
}

int qs_probs_n(qs_handle_t h, const void* states, int64_t n_amps, float* probs) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(states && ((uintptr_t)states & 15u) == 0, "states must be a 16-byte aligned device pointer");
  QS_CHECK_ARG(probs != nullptr && ((uintptr_t)probs & 7u) == 0, "probs must be a non-null 8-byte aligned pointer");
  QS_CHECK_ARG(n_amps >= 0 && (n_amps & 1) == 0, "n_amps must be even and >= 0");
  const uint64_t nvec = (uint64_t)n_amps / 2;
  if (nvec) {
    qs_launch_pdl(h, k_probs, dim3(qs_blocks_for(h, nvec, kThreads)), dim3(kThreads), 0, (const float4*)states, (float2*)probs, nvec);
    qs_after_launch(h, "k_probs");
  }
  QS_API_END(h)
}

int qs_measure(qs_handle_t h, void* state, int n, int t, double u, int* outcome) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(t, n, "target");
  QS_CHECK_ARG(outcome != nullptr, "outcome is null");
  double* o = red_out(h);
  const uint64_t nvec = (1ull << n) / 2;
  reduce_to(h, FP0{(const float4*)state, t}, nvec, o, 0, red_part(h));
  // the kernel writes the outcome straight into the handle's pinned buffer
  // (page-locked host memory is addressable from the device under unified
  // addressing), so no copy is queued between the kernel and the synchronise
  int* pin = reinterpret_cast<int*>(h->pinned_get(64));
  qs_launch_pdl(h, k_collapse, dim3(qs_blocks_for(h, nvec, kThreads)), dim3(kThreads), 0, (float4*)state, nvec, t, u, o, pin);
  qs_after_launch(h, "k_collapse");
  QS_CUDA(cudaStreamSynchronize(h->stream));
  *outcome = *pin;
  QS_API_END(h)
}

int qs_expect_z(qs_handle_t h, const void* state, int n, uint64_t zmask, double* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(out != nullptr, "out is null");
  double* o = red_out(h);
  reduce_to(h, FZ{(const float4*)state, zmask}, (1ull << n) / 2, o, 0, red_part(h));
  *out = fetch_scalar(h, o);
  QS_API_END(h)
}

int qs_expect_pauli_sum(qs_handle_t h, const void* state, int n, const uint64_t* x, const uint64_t* z,
                        const double* c, int nterms, double* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(out != nullptr, "out is null");
  QS_CHECK_ARG(nterms >= 1 && nterms <= 1024, "n_terms must be in [1, 1024]");
  const size_t toff = 64 + 8 * kMaxBlocks;
  Term* dT = (Term*)qs_upload_terms(h, toff, n, x, z, c, nterms);
  double* o = red_out(h);
  double* part = red_part(h);
  const uint64_t N = 1ull << n;
  Slicing sl = slice(N);
  qs_launch_pdl(h, k_pauli_expect, dim3(sl.nb), dim3(kThreads), sizeof(Term) * nterms, (const float2*)state, N, dT, nterms, sl.per,
                                                                        part);
  qs_after_launch(h, "k_pauli_expect");
  qs_launch_pdl(h, k_final, dim3(1), dim3(1024), 0, part, sl.nb, o, 0);
  qs_after_launch(h, "k_final");
  *out = fetch_scalar(h, o);
  QS_API_END(h)
}

int qs_apply_pauli_sum(qs_handle_t h, const void* psi, void* out, int n, const uint64_t* x, const uint64_t* z,
                       const double* c, int nterms) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(psi, n);
  qs_check_state(out, n);
  QS_CHECK_ARG(psi != out, "out must not alias psi");
  QS_CHECK_ARG(nterms >= 1 && nterms <= 1024, "n_terms must be in [1, 1024]");
  Term* dT = (Term*)qs_upload_terms(h, 0, n, x, z, c, nterms);
  const uint64_t N = 1ull << n;
  qs_launch_pdl(h, k_pauli_apply, dim3(qs_blocks_for(h, N, kThreads)), dim3(kThreads), sizeof(Term) * nterms, 
      (const float2*)psi, (float2*)out, N, dT, nterms);
  qs_after_launch(h, "k_pauli_apply");
  QS_API_END(h)
}


// Per device, once: the scan kernels' shared-memory limit raised to their
// tile, and the chunk-sum kernels' grids sized to one wave of the CTAs that
// fit on an SM at once (registers and 34 KiB of staging each decide how many),
// so that no second wave runs on part of the SMs while the rest idle.
struct SampleLaunch {
  int sums_per_sm, sums_b_per_sm;
};
static SampleLaunch sample_launch(qs_context* h) {
  static std::mutex mu;
  static std::map<int, SampleLaunch> by_device;
  std::lock_guard<std::mutex> lk(mu);
  auto f = by_device.find(h->device);
  if (f != by_device.end()) return f->second;
  QS_CUDA(cudaFuncSetAttribute(k_chunk_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScanSmem));
  QS_CUDA(cudaFuncSetAttribute(k_chunk_scan_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScanSmem));
  SampleLaunch L{0, 0};
  QS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&L.sums_per_sm, k_chunk_sums, kThreads, 0));
  QS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&L.sums_b_per_sm, k_chunk_sums_b, kThreads, 0));
  if (L.sums_per_sm < 1 || L.sums_b_per_sm < 1) throw qs_error(QS_ERR_CUDA, "chunk-sum kernel does not fit on an SM");
  by_device[h->device] = L;
  return L;
}

int qs_sample_batched(qs_handle_t h, const void* states, int n_states, const int32_t* widths,
                      const int64_t* state_offsets, const int64_t* shots, const uint64_t* seeds, int64_t* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(n_states >= 0, "n_states must be >= 0");
  if (n_states == 0) return QS_OK;
  QS_CHECK_ARG(states && widths && state_offsets && shots && seeds, "null batch descriptor");
  QS_CHECK_ARG(((uintptr_t)states & 15u) == 0, "states must be 16-byte aligned");
  // descriptors, plus one sentinel holding the totals
  std::vector<SampleDesc> desc(n_states + 1);
  uint64_t chunks = 0, nshots = 0;
  for (int t = 0; t < n_states; ++t) {
    QS_CHECK_ARG(widths[t] >= 1 && widths[t] <= QS_MAX_QUBITS, "state width out of range");
    QS_CHECK_ARG(state_offsets[t] >= 0 && shots[t] >= 0, "negative offset or shot count");
    const uint64_t N = 1ull << widths[t];
    SampleDesc& D = desc[t];
    D.state_off = (uint64_t)state_offsets[t];
    D.n = N;
    D.nchunks = (N + kChunk - 1) / kChunk;
    D.chunk_off = chunks;
    D.shot_off = nshots;
    D.seed = seeds[t];
    chunks += D.nchunks;
    nshots += (uint64_t)shots[t];
  }
  desc[n_states] = SampleDesc{0, 0, 0, chunks, nshots, 0};
  if (nshots == 0) return QS_OK;
  QS_CHECK_ARG(out != nullptr, "out pointer is null");
  const size_t dbytes = ((desc.size() * sizeof(SampleDesc)) + 255) & ~size_t(255);
  char* sc = static_cast<char*>(h->scratch_get(dbytes + sizeof(double) * (2 * chunks + n_states)));
  auto* d_desc = reinterpret_cast<SampleDesc*>(sc);
  double* csum = reinterpret_cast<double*>(sc + dbytes);
  double* cbase = csum + chunks;
  QS_CUDA(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(SampleDesc), cudaMemcpyHostToDevice, h->stream));
  const int wpb = kThreads / 32;
  const SampleLaunch L = sample_launch(h);
  qs_launch_pdl(h, k_chunk_sums_b, dim3(qs_blocks_for(h, chunks * 32, kThreads, L.sums_b_per_sm)), dim3(kThreads), 0, 
      (const float2*)states, d_desc, n_states, chunks, csum);
  qs_after_launch(h, "k_chunk_sums_b");
  qs_launch_pdl(h, k_chunk_scan_b, dim3((unsigned)n_states), dim3(kScanThreads), kScanSmem, csum, d_desc, cbase);
  qs_after_launch(h, "k_chunk_scan_b");
  const uint64_t blocks = std::min<uint64_t>((nshots + wpb - 1) / wpb, (uint64_t)h->sm_count * 16);
  qs_launch_pdl(h, k_sample_b, dim3((unsigned)blocks), dim3(kThreads), 0, (const float2*)states, d_desc, n_states, nshots, cbase,
                                                           out);
  qs_after_launch(h, "k_sample_b");
  QS_API_END(h)
}

int qs_sample(qs_handle_t h, const void* state, int n, const double* u, int64_t nshots, int64_t* out) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  QS_CHECK_ARG(nshots >= 0, "n_shots must be >= 0");
  if (nshots == 0) return QS_OK;
  QS_CHECK_ARG(u != nullptr && out != nullptr, "u/out pointer is null");
  const uint64_t N = 1ull << n;
  const uint64_t nchunks = (N + kChunk - 1) / kChunk;
  double* base = (double*)h->scratch_get(sizeof(double) * (2 * nchunks + 1));
  double* csum = base;
  double* cbase = base + nchunks;
  const int wpb = kThreads / 32;
  const SampleLaunch L = sample_launch(h);
  qs_launch_pdl(h, k_chunk_sums, dim3(qs_blocks_for(h, nchunks * 32, kThreads, L.sums_per_sm)), dim3(kThreads), 0, (const float2*)state, N,
                                                                                     nchunks, csum);
  qs_after_launch(h, "k_chunk_sums");
  qs_launch_pdl(h, k_chunk_scan, dim3(1), dim3(kScanThreads), kScanSmem, csum, nchunks, cbase);
  qs_after_launch(h, "k_chunk_scan");
  const uint64_t blocks = std::min<uint64_t>(((uint64_t)nshots + wpb - 1) / wpb, (uint64_t)h->sm_count * 16);
  qs_launch_pdl(h, k_sample, dim3((unsigned)blocks), dim3(kThreads), 0, (const float2*)state, N, nchunks, cbase, u, nshots, out);
  qs_after_launch(h, "k_sample");
  QS_API_END(h)
}

}  // extern "C"
