// Stable LSD radix sort of (64-bit key, 32-bit value) pairs and a three-phase
// int scan, the two device-wide primitives of the plan builder (sort of the
// samples by tile / CF / position key, tile item offsets, run ends and the
// degrid write-back order).
//
// Sort, per 8-bit digit pass (reduce-then-scan, as in Merrill and Grimshaw's
// "High performance and scalable radix sorting", 2011):
//   k_sort_upsweep    one CTA per contiguous segment of 4096-key tiles:
//                     the segment's digit histogram (warp-aggregated shared
//                     atomics), stored digit-major: counts[d * nseg + seg].
//   k_sort_scan       one CTA: exclusive scan of counts, so that
//                     counts[d * nseg + seg] becomes the global output
//                     position of the segment's first key of digit d.
//   k_sort_downsweep  the same segments, tile by tile in order: each warp
//                     ranks its 512 keys (16 per lane, index order
//                     item-major then lane) by digit with __match_any_sync
//                     and per-warp digit counters; warp prefixes and the
//                     tile's digit starts give every key its place in a
//                     shared-memory copy of the tile sorted by digit, which
//                     is written out in order (runs of equal digits are
//                     contiguous in the output).  Ranks follow input order
//                     inside a warp, warps in order inside a tile and tiles
//                     in order inside a segment, so each pass is stable.
// Only bits [0, end_bit) order the keys (the last pass masks the bits above).
// Keys past n in the last tile are all ones (the largest digit, after every
// valid key of the tile) and are not written.
//
// Scan: k_scan_reduce (one partial per segment of 2048-element chunks),
// k_scan_parts (exclusive scan of the partials), k_scan_apply (each segment
// rescanned from its carry, four elements per thread).
#include "yg_sort.h"

#include <algorithm>
#include <atomic>
#include <climits>

namespace yg {

extern std::atomic<long long> g_kernel_launches;
#define YG_SORT_COUNT() g_kernel_launches.fetch_add(1, std::memory_order_relaxed)

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortIpt = 16;
constexpr int kSortTile = kSortThreads * kSortIpt;  // 4096 keys
constexpr int kDigits = 256;
constexpr int kSortSegPerSm = 2;  // two downsweep CTAs fit an SM (128 registers a thread)
constexpr size_t kDownSmem = (size_t)kSortTile * 8 + (size_t)kSortTile * 4 + (size_t)kSortWarps * kDigits * 4 +
                             3 * kDigits * 4 + 64;

constexpr int kScanThreads = 512;
constexpr int kScanIpt = 4;
constexpr int kScanChunk = kScanThreads * kScanIpt;  // 2048 elements
constexpr int kScanSegPerSm = 4;

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, sms);
}

struct SortGeom {
  long long ntiles;
  int nseg;
};

SortGeom sort_geom(long long n) {
  SortGeom g;
  g.ntiles = (n + kSortTile - 1) / kSortTile;
  g.nseg = (int)std::max(1ll, std::min<long long>(g.ntiles, (long long)sm_count() * kSortSegPerSm));
  return g;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_upsweep(const unsigned long long* __restrict__ keys,
                                                               long long n, int shift, unsigned dmask,
                                                               long long ntiles, int nseg,
                                                               unsigned* __restrict__ counts) {
  __shared__ unsigned hist[kSortWarps][kDigits];
  const int tid = threadIdx.x, w = tid >> 5;
  for (int i = tid; i < kSortWarps * kDigits; i += kSortThreads) (&hist[0][0])[i] = 0u;
  __syncthreads();
  const int seg = blockIdx.x;
  const long long i0 = ntiles * seg / nseg * kSortTile;
  const long long i1 = std::min(n, ntiles * (seg + 1) / nseg * kSortTile);
  const unsigned lt = lanemask_lt();
  for (long long c = i0; c < i1; c += 4 * kSortThreads) {
    unsigned d[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long i = c + q * kSortThreads + tid;
      d[q] = i < i1 ? (unsigned)(keys[i] >> shift) & dmask : 256u;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const unsigned peers = __match_any_sync(0xffffffffu, d[q]);
      if (d[q] < 256u && (peers & lt) == 0u) atomicAdd(&hist[w][d[q]], (unsigned)__popc(peers));
    }
  }
  __syncthreads();
  for (int dg = tid; dg < kDigits; dg += kSortThreads) {
    unsigned s = 0;
#pragma unroll
    for (int ww = 0; ww < kSortWarps; ++ww) s += hist[ww][dg];
    counts[(size_t)dg * nseg + seg] = s;
  }
}

// exclusive scan of m counts by one CTA of 1024 threads, in place
__global__ void __launch_bounds__(1024) k_sort_scan(unsigned* __restrict__ counts, int m) {
  __shared__ unsigned part[1024];
  const int tid = threadIdx.x;
  const int per = (m + 1023) / 1024;
  const int b0 = std::min(m, tid * per), b1 = std::min(m, b0 + per);
  unsigned s = 0;
  for (int i = b0; i < b1; ++i) s += counts[i];
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned v = tid >= off ? part[tid - off] : 0u;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  unsigned run = part[tid] - s;
  for (int i = b0; i < b1; ++i) {
    const unsigned c = counts[i];
    counts[i] = run;
    run += c;
  }
}

__global__ void __launch_bounds__(kSortThreads) k_sort_downsweep(const unsigned long long* __restrict__ kin,
                                                                 const unsigned* __restrict__ vin,
                                                                 unsigned long long* __restrict__ kout,
                                                                 unsigned* __restrict__ vout, long long n, int shift,
                                                                 unsigned dmask, long long ntiles, int nseg,
                                                                 const unsigned* __restrict__ offsets) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* sk = reinterpret_cast<unsigned long long*>(smem);
  unsigned* sv = reinterpret_cast<unsigned*>(sk + kSortTile);
  unsigned* whist = sv + kSortTile;           // [warp][digit]
  unsigned* tstart = whist + kSortWarps * kDigits;
  unsigned* tcount = tstart + kDigits;
  unsigned* run = tcount + kDigits;           // output position of the next key of each digit
  unsigned* wsum = run + kDigits;             // 8 warp totals
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int seg = blockIdx.x;
  const unsigned lt = lanemask_lt();
  run[tid] = offsets[(size_t)tid * nseg + seg];  // kSortThreads == kDigits
  const long long t0 = ntiles * seg / nseg, t1 = ntiles * (seg + 1) / nseg;
  unsigned* wh = whist + w * kDigits;
  for (long long t = t0; t < t1; ++t) {
    const long long base = t * kSortTile;
    const int nvalid = (int)std::min<long long>(kSortTile, n - base);
    for (int i = tid; i < kSortWarps * kDigits; i += kSortThreads) whist[i] = 0u;
    __syncthreads();
    unsigned long long k[kSortIpt];
    unsigned v[kSortIpt], rk[kSortIpt];
    const int wbase = w * 32 * kSortIpt;
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
      const int j = wbase + i * 32 + lane;
      if (j < nvalid) {
        k[i] = kin[base + j];
        v[i] = vin[base + j];
      } else {
        k[i] = ~0ull;
        v[i] = 0u;
      }
    }
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
      const unsigned d = (unsigned)(k[i] >> shift) & dmask;
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const unsigned before = wh[d];
      __syncwarp();
      if ((peers & lt) == 0u) wh[d] = before + (unsigned)__popc(peers);
      __syncwarp();
      rk[i] = before + (unsigned)__popc(peers & lt);
    }
    __syncthreads();
    {
      // per digit: exclusive prefix over warps, and the tile's count
      unsigned s = 0;
#pragma unroll
      for (int ww = 0; ww < kSortWarps; ++ww) {
        const unsigned c = whist[ww * kDigits + tid];
        whist[ww * kDigits + tid] = s;
        s += c;
      }
      tcount[tid] = s;
      unsigned x = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[w] = x;
      __syncthreads();
      unsigned pre = 0;
      for (int ww = 0; ww < w; ++ww) pre += wsum[ww];
      tstart[tid] = pre + x - s;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSortIpt; ++i) {
      const unsigned d = (unsigned)(k[i] >> shift) & dmask;
      const unsigned p = tstart[d] + wh[d] + rk[i];
      sk[p] = k[i];
      sv[p] = v[i];
    }
    __syncthreads();
    for (int j = tid; j < nvalid; j += kSortThreads) {
      const unsigned long long key = sk[j];
      const unsigned d = (unsigned)(key >> shift) & dmask;
      const unsigned o = run[d] + (unsigned)j - tstart[d];
      kout[o] = key;
      vout[o] = sv[j];
    }
    __syncthreads();
    run[tid] += tcount[tid] - ((unsigned)tid == dmask ? (unsigned)(kSortTile - nvalid) : 0u);
    __syncthreads();
  }
}

template <int OP>
__device__ __forceinline__ int sop(int a, int b) {
  if (OP == SCAN_SUM) return a + b;
  if (OP == SCAN_MIN) return a < b ? a : b;
  return a > b ? a : b;
}

template <int OP>
__host__ __device__ constexpr int sident() {
  return OP == SCAN_SUM ? 0 : (OP == SCAN_MIN ? INT_MAX : INT_MIN);
}

struct ScanGeom {
  long long nchunks;
  int nseg;
};

ScanGeom scan_geom(long long n) {
  ScanGeom g;
  g.nchunks = (n + kScanChunk - 1) / kScanChunk;
  g.nseg = (int)std::max(1ll, std::min<long long>(g.nchunks, std::min(1024, sm_count() * kScanSegPerSm)));
  return g;
}

// the four elements of thread tid in chunk c (identity past n)
__device__ __forceinline__ void scan_load4(const int* __restrict__ in, long long n, long long c, int tid, int idv,
                                           bool vec, int x[4]) {
  const long long i = c * kScanChunk + (long long)tid * kScanIpt;
  if (vec && i + 3 < n) {
    const int4 q = *reinterpret_cast<const int4*>(in + i);
    x[0] = q.x;
    x[1] = q.y;
    x[2] = q.z;
    x[3] = q.w;
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) x[e] = i + e < n ? in[i + e] : idv;
  }
}

// block-wide exclusive scan of one value per thread; *total gets the op over all
template <int OP>
__device__ __forceinline__ int block_excl(int x, int* wtot, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc = sop<OP>(y, inc);
  }
  if (lane == 31) wtot[w] = inc;
  __syncthreads();
  int pre = sident<OP>(), all = sident<OP>();
  for (int ww = 0; ww < kScanThreads / 32; ++ww) {
    if (ww < w) pre = sop<OP>(pre, wtot[ww]);
    all = sop<OP>(all, wtot[ww]);
  }
  __syncthreads();
  *total = all;
  const int excl_in_warp = __shfl_up_sync(0xffffffffu, inc, 1);
  return lane == 0 ? pre : sop<OP>(pre, excl_in_warp);
}

template <int OP>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ in, long long n,
                                                              long long nchunks, int nseg, bool vec,
                                                              int* __restrict__ part) {
  __shared__ int wtot[kScanThreads / 32];
  const int seg = blockIdx.x;
  const long long c0 = nchunks * seg / nseg, c1 = nchunks * (seg + 1) / nseg;
  int acc = sident<OP>();
  for (long long c = c0; c < c1; ++c) {
    int x[4];
    scan_load4(in, n, c, threadIdx.x, sident<OP>(), vec, x);
    acc = sop<OP>(acc, sop<OP>(sop<OP>(x[0], x[1]), sop<OP>(x[2], x[3])));
  }
  int total;
  block_excl<OP>(acc, wtot, &total);
  if (threadIdx.x == 0) part[seg] = total;
}

template <int OP>
__global__ void __launch_bounds__(1024) k_scan_parts(int* __restrict__ part, int nseg) {
  __shared__ int buf[1024];
  const int tid = threadIdx.x;
  buf[tid] = tid < nseg ? part[tid] : sident<OP>();
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = tid >= off ? buf[tid - off] : sident<OP>();
    __syncthreads();
    buf[tid] = sop<OP>(v, buf[tid]);
    __syncthreads();
  }
  if (tid < nseg) part[tid] = tid == 0 ? sident<OP>() : buf[tid - 1];
}

template <int OP>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int* in, int* out, long long n,
                                                             long long nchunks, int nseg, bool vec, bool exclusive,
                                                             const int* __restrict__ part) {
  __shared__ int wtot[kScanThreads / 32];
  const int seg = blockIdx.x;
  const long long c0 = nchunks * seg / nseg, c1 = nchunks * (seg + 1) / nseg;
  int carry = part[seg];
  for (long long c = c0; c < c1; ++c) {
    int x[4];
    scan_load4(in, n, c, threadIdx.x, sident<OP>(), vec, x);
    const int tot4 = sop<OP>(sop<OP>(x[0], x[1]), sop<OP>(x[2], x[3]));
    int btotal;
    const int ex = block_excl<OP>(tot4, wtot, &btotal);
    int run = sop<OP>(carry, ex);
    int y[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int incl = sop<OP>(run, x[e]);
      y[e] = exclusive ? run : incl;
      run = incl;
    }
    const long long i = c * kScanChunk + (long long)threadIdx.x * kScanIpt;
    if (vec && i + 3 < n) {
      *reinterpret_cast<int4*>(out + i) = make_int4(y[0], y[1], y[2], y[3]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (i + e < n) out[i + e] = y[e];
    }
    carry = sop<OP>(carry, btotal);
  }
}

template <int OP>
cudaError_t scan_launch(const int* in, int* out, long long n, bool exclusive, int* part, cudaStream_t st) {
  const ScanGeom g = scan_geom(n);
  const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
  k_scan_reduce<OP><<<g.nseg, kScanThreads, 0, st>>>(in, n, g.nchunks, g.nseg, vec, part);
  YG_SORT_COUNT();
  k_scan_parts<OP><<<1, 1024, 0, st>>>(part, g.nseg);
  YG_SORT_COUNT();
  k_scan_apply<OP><<<g.nseg, kScanThreads, 0, st>>>(in, out, n, g.nchunks, g.nseg, vec, exclusive, part);
  YG_SORT_COUNT();
  return cudaGetLastError();
}

}  // namespace

size_t sort_pairs_tmp_bytes(long long n) {
  const SortGeom g = sort_geom(std::max(1ll, n));
  return (size_t)kDigits * g.nseg * sizeof(unsigned);
}

cudaError_t sort_pairs(unsigned long long* k0, unsigned long long* k1, unsigned int* v0, unsigned int* v1,
                       long long n, int end_bit, void* tmp, size_t tmp_bytes, cudaStream_t st, int* in_alt) {
  *in_alt = 0;
  if (n <= 1 || end_bit <= 0) return cudaSuccess;
  if (n >= (1ll << 31) || end_bit > 64) return cudaErrorInvalidValue;
  const SortGeom g = sort_geom(n);
  if (tmp_bytes < (size_t)kDigits * g.nseg * sizeof(unsigned)) return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_sort_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDownSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  unsigned* counts = static_cast<unsigned*>(tmp);
  unsigned long long* ks[2] = {k0, k1};
  unsigned* vs[2] = {v0, v1};
  int cur = 0;
  for (int shift = 0; shift < end_bit; shift += 8) {
    const unsigned dmask = end_bit - shift >= 8 ? 255u : (1u << (end_bit - shift)) - 1u;
    k_sort_upsweep<<<g.nseg, kSortThreads, 0, st>>>(ks[cur], n, shift, dmask, g.ntiles, g.nseg, counts);
    YG_SORT_COUNT();
    k_sort_scan<<<1, 1024, 0, st>>>(counts, kDigits * g.nseg);
    YG_SORT_COUNT();
    k_sort_downsweep<<<g.nseg, kSortThreads, kDownSmem, st>>>(ks[cur], vs[cur], ks[cur ^ 1], vs[cur ^ 1], n, shift,
                                                              dmask, g.ntiles, g.nseg, counts);
    YG_SORT_COUNT();
    cur ^= 1;
  }
  *in_alt = cur;
  return cudaGetLastError();
}

size_t scan_tmp_bytes(long long n) { return (size_t)scan_geom(std::max(1ll, n)).nseg * sizeof(int); }

cudaError_t scan_i32(const int* in, int* out, long long n, int op, bool exclusive, void* tmp, size_t tmp_bytes,
                     cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (n >= (1ll << 31)) return cudaErrorInvalidValue;
  if (tmp_bytes < scan_tmp_bytes(n)) return cudaErrorInvalidValue;
  int* part = static_cast<int*>(tmp);
  switch (op) {
    case SCAN_SUM: return scan_launch<SCAN_SUM>(in, out, n, exclusive, part, st);
    case SCAN_MIN: return scan_launch<SCAN_MIN>(in, out, n, exclusive, part, st);
    case SCAN_MAX: return scan_launch<SCAN_MAX>(in, out, n, exclusive, part, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace yg
