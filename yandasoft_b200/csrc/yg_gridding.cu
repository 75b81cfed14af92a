// Binning, tiled gridding and degridding kernels of the B200 gridder.
//
// Pipeline of one grid (or degrid) pass over a chunk of visibilities:
//   k_bin          one thread per (row, chan) sample: FP64 bit-exact uv cell,
//                  oversample offsets, w-plane, CF index, strict on-grid test
//                  (TableVisGridder.cc:604-764), and a 64-bit sort key
//                  (grid plane, image channel, uv tile, CF index, Morton
//                  position inside the tile; or, for a gridding-only plan of
//                  the plane-major kernel, tile, CF plane, position, offset).
//   radix sort     stable LSD radix sort of (key, sample id) (yg_sort.cu).
//   k_tile_bounds  start/end of every tile's run in the sorted list.
//   work items     tiles split into items of at most vmax samples.
//   k_records      one 16-byte record per sorted sample (footprint origin,
//                  residues, CF width and index, sample id).
//   k_sum_weights  weight checks and sums of weights over the sorted records.
//   k_grid         one CTA per item over CF-major records: the padded tile
//                  (T + 2 Smax)^2 lives in shared memory; every thread owns
//                  the cells of a fixed residue class (x mod W, y mod W), so no
//                  two threads ever touch the same cell (no atomics); its
//                  weighted visibilities come from k_gather_cube.
//   k_grid_pl      the same over plane-major records, each CF plane's
//                  oversampling offsets staged in shared memory once, running
//                  sums in registers, the tile in shared or global memory; its
//                  producer warp forms the weighted visibilities itself.
//   k_halo_sum     each output tile adds, in a fixed order, the overlapping
//                  parts of its neighbours' padded tiles: deterministic, and
//                  the grid is written once.
//   k_degrid_r     16-wide CFs: one CTA per item, the padded grid tile in
//                  shared memory, a warp per segment with its CF column in
//                  registers, two samples per half-warp pass.
//   k_degrid_t     wider CFs (and the learned forms): the CF plane per tap
//                  from the ring, transposing warp-shuffle reductions.
//   k_degrid_writeback  the reference's write-back semantics, including the
//                  value it carries into off-grid samples.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "yg_internal.h"
#include "yg_mlp.cuh"
#include "yg_sort.h"

namespace yg {

// number of this library's own kernel launches
std::atomic<long long> g_kernel_launches{0};
#define YG_COUNT_LAUNCH() g_kernel_launches.fetch_add(1, std::memory_order_relaxed)


__device__ __forceinline__ unsigned int morton2(unsigned int x, unsigned int y) {
  auto spread = [](unsigned int v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

// ---------------------------------------------------------------------------
// k_bin
// status: 0 = not used (flagged / unmapped / rejected row), 1 = w out of range
// (clipped), 2 = valid but off the grid, 3 = gridded/degridded.
// ---------------------------------------------------------------------------
__global__ void k_bin(BinArgs a, unsigned long long* __restrict__ key, unsigned int* __restrict__ val,
                      unsigned int* __restrict__ pos, int* __restrict__ cfi_out,
                      unsigned char* __restrict__ status, DevError* err) {
  const long long n = a.nrow * (long long)a.nchan;
  const long long ntiles = (long long)a.ntx * a.nty;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const long long row = s % a.nrow;
    const int chan = (int)(s / a.nrow);
    unsigned long long k = a.invalid_key;
    unsigned int p = 0;
    int cfi = 0;
    unsigned char st = 0;
    if (!a.row_ok || a.row_ok[row]) {
      const double f = a.freq[chan];
      const double u = a.uvw[3 * row + 0], v = a.uvw[3 * row + 1], w = a.uvw[3 * row + 2];
      int iu, iv, fu, fv;
      if (!axis_index(f, u, a.cellu, a.os, a.nx, &iu, &fu) || !axis_index(f, v, a.cellv, a.os, a.ny, &iv, &fv)) {
        raise_error(err, YG_ERR_FRAC, s);
      } else {
        // w-plane indices are computed for every sample, as initIndices does
        int e = 0, plane = 0, gind = 0;
        if (a.cf_mode != CF_MODE_SINGLE || a.grid_mode != GRID_MODE_SINGLE) {
          const double wf = __dmul_rn(__ddiv_rn(w, kC), f);
          if (a.cf_mode == CF_MODE_WSTACK_WPROJ) {
            gind = get_wplane(a.ws_stack, wf, &e);
            if (gind >= 0) {
              const int half = (a.ws_stack.nwplanes - 1) / 2;
              const double wst = __dmul_rn((double)(gind - half), a.ws_stack.wscale);
              plane = get_wplane(a.ws, __dsub_rn(wf, wst), &e);
            } else {
              plane = -1;
            }
          } else {
            plane = get_wplane(a.ws, wf, &e);
            gind = (a.grid_mode == GRID_MODE_WPLANE) ? plane : 0;
          }
          if (e) raise_error(err, e, s);
        }
        int cplane = 0;
        if (a.cf_mode == CF_MODE_WPLANE || a.cf_mode == CF_MODE_WSTACK_WPROJ) {
          cplane = plane;
        } else if (a.cf_mode == CF_MODE_AW) {
          const int fd = a.feed ? a.feed[row] : 0;
          cplane = plane;
          if (plane >= 0) {
            const int c = a.aw_nchan > 1 ? chan : 0;
            cplane = plane + a.ws.nwplanes * (c + a.aw_nchan * (fd + a.aw_maxfeeds * a.aw_field));
          }
        }
        bool good = true;
        if (a.flag) {
          for (int pol = 0; pol < a.npol; ++pol) {
            if (a.flag[s + n * pol]) { good = false; break; }
          }
        }
        const int ichan = a.chan_map[chan];
        if (good && ichan >= 0) {
          if (gind < 0 || cplane < 0) {
            st = 1;
          } else {
            cfi = fu + a.os * (fv + a.os * cplane);
            if (cfi < 0 || cfi >= a.cf.ncf || a.cf.size[cfi] <= 0) {
              raise_error(err, YG_ERR_CINDEX, s);
            } else {
              const int support = (a.cf.size[cfi] - 1) / 2;
              int offu = 0, offv = 0;
              if (a.cf.offsets && cplane < a.cf.noffsets) {
                const int2 o = a.cf.offsets[cplane];
                offu = o.x;
                offv = o.y;
              }
              const int iuo = iu + offu, ivo = iv + offv;
              if ((iuo - support) > 0 && (ivo - support) > 0 && (iuo + support) < a.nx && (ivo + support) < a.ny) {
                st = 3;
                const int tx = iuo / a.tile, ty = ivo / a.tile;
                const long long tile = tx + (long long)a.ntx * ty;
                const long long gc = (long long)gind * a.nchan_img + ichan;
                const unsigned int m = morton2((unsigned)(iuo - tx * a.tile), (unsigned)(ivo - ty * a.tile));
                if (a.key_planes) {
                  // plane-major: tile, CF plane, position, oversampling offset
                  const unsigned long long os2 = (unsigned long long)a.os * a.os;
                  const unsigned long long cp = (unsigned)cfi / os2, fr = (unsigned)cfi % os2;
                  k = (((((unsigned long long)(gc * ntiles + tile) * ((unsigned long long)a.cf.ncf / os2) + cp)
                         << a.mbits) | m) * os2) + fr;
                } else {
                  k = (((unsigned long long)(gc * ntiles + tile) * (unsigned long long)a.cf.ncf + (unsigned)cfi)
                       << a.mbits) | m;
                }
                p = (unsigned)iuo | ((unsigned)ivo << 16);
              } else {
                st = 2;
              }
            }
          }
        }
      }
    }
    key[s] = k;
    val[s] = (unsigned int)s;
    pos[s] = p;
    cfi_out[s] = cfi;
    status[s] = st;
  }
}

// tile id of a sorted key: ((tile * ncf + cfi) << mbits) | morton, or with
// kos2 = os^2 the plane-major key of a gridding-only plan,
// ((((tile * ncp + plane) << mbits) | morton) * os^2 + offset), ncp = ncf / os^2
__device__ __forceinline__ long long key_tile(unsigned long long k, int mbits, int ncf, int kos2) {
  return (long long)(((k / (unsigned long long)kos2) >> mbits) / (unsigned long long)(ncf / kos2));
}

__global__ void k_tile_bounds(const unsigned long long* __restrict__ key, long long n, int mbits, int ncf, int kos2,
                              unsigned long long invalid_key, int* __restrict__ tstart, int* __restrict__ tend,
                              long long* nvalid) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = key[i];
    if (k >= invalid_key) continue;
    const long long t = key_tile(k, mbits, ncf, kos2);
    if (i == 0 || key_tile(key[i - 1], mbits, ncf, kos2) != t) tstart[t] = (int)i;
    const bool last = (i == n - 1) || key[i + 1] >= invalid_key;
    if (last || key_tile(key[i + 1], mbits, ncf, kos2) != t) tend[t] = (int)(i + 1);
    if (last) *nvalid = i + 1;
  }
}

__global__ void k_count_items(const int* __restrict__ tstart, const int* __restrict__ tend, long long ntiles,
                              int vmax, int* __restrict__ nit) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles; t += (long long)gridDim.x * blockDim.x) {
    const int c = tend[t] - tstart[t];
    nit[t] = c > 0 ? (c + vmax - 1) / vmax : 0;
  }
}

__global__ void k_fill_items(const int* __restrict__ tstart, const int* __restrict__ tend,
                             const int* __restrict__ nit, const int* __restrict__ base, long long ntiles, int vmax,
                             int4* __restrict__ items) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles; t += (long long)gridDim.x * blockDim.x) {
    const int m = nit[t];
    const int b = base[t];
    for (int j = 0; j < m; ++j) {
      const int s0 = tstart[t] + j * vmax;
      const int s1 = min(tend[t], s0 + vmax);
      items[b + j] = make_int4((int)t, s0, s1, 0);
    }
  }
}

// ---------------------------------------------------------------------------
// weights: rVis = phasor * conj(vis) * wt (* mfs), TableVisGridder.cc:775-806
// ---------------------------------------------------------------------------
__device__ __forceinline__ float noise_weight(float nre) {
  const float vn = __fmul_rn(nre, nre);
  return (vn > 0.f) ? (float)(1.0 / (double)vn) : 0.f;
}

__device__ __forceinline__ void phasor_of(const VisArgs& v, long long row, int chan, float* pr, float* pi) {
  if (!v.delay) {
    *pr = 1.f;
    *pi = 0.f;
    return;
  }
  const double ph = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, kPi), v.freq[chan]), v.delay[row]), kC);
  *pr = (float)cos(ph);
  *pi = (float)sin(ph);
}

// rVis = phasor * conj(vis) * wt (* mfs) of sample s, polarisation p
// (TableVisGridder.cc:775-806), wt (* mfs) for the PSF, wt for the
// preconditioner function; FP32 with explicit rounding.
__device__ __forceinline__ float2 weighted_vis(const VisArgs& v, long long s, long long n, int p, float pr, float pi,
                                               float m) {
  const float nre = v.noise ? v.noise[s + n * p].x : 1.f;
  const float wt = noise_weight(nre);
  if (v.pcf) return make_float2(__fmul_rn(1.f, wt), __fmul_rn(0.f, wt));
  if (v.psf) return make_float2(__fmul_rn(__fmul_rn(1.f, wt), m), __fmul_rn(__fmul_rn(0.f, wt), m));
  const float2 vv = v.vis[s + n * p];
  const float vr = vv.x, vi = -vv.y;
  float rr = __fsub_rn(__fmul_rn(pr, vr), __fmul_rn(pi, vi));
  float ri = __fadd_rn(__fmul_rn(pr, vi), __fmul_rn(pi, vr));
  rr = __fmul_rn(__fmul_rn(rr, wt), m);
  ri = __fmul_rn(__fmul_rn(ri, wt), m);
  return make_float2(rr, ri);
}


// ---------------------------------------------------------------------------
// k_grid
// ---------------------------------------------------------------------------
struct GridKArgs {
  const int4* items;
  const unsigned int* val;   // sample ids, sorted
  const int4* rec;           // per sorted sample: cell, residues|w, cf index, sample id
  const float2* svis;        // per sorted sample: npol weighted visibilities (k_grid_pl: null,
                             // its producer forms them from the cube itself)
  const unsigned int* pos;   // iu | iv << 16, unsorted (by sample id)
  const int* cfi;            // unsorted
  VisArgs v;
  CFView cf;
  int tile, ntx;
  long long ntiles;
  int smax;                  // Smax of the plan
  int P;                     // T + 2 Smax: the padded tile written to scratch
  int Pg;                    // row stride of the shared-memory tile, P plus a gutter
  int Wp;                    // residue modulus: round_up(2 Smax + 1, 16)
  int cfbuf;                 // bytes of one shared-memory CF buffer
  float2* scratch;           // [item][npol][P][P]
  int pol0;                  // first polarisation of this pass
  int npol_total;            // polarisations of the visibility cube
  int stage_bytes;           // bytes of one segment stage
  int nstages;               // depth of the segment ring
  int pps;                   // CF planes (runs) per stage, CFM 0
  int cfplane;               // bytes of one CF plane slot
  int Wy;                    // row modulus of the residues (the plan's)
  int pos_major;             // records in position-major order, taps read through L2
  LearnedCF lcf;             // the network of the learned CF mode
  const float4* ext;         // continuous learned CF: per sorted sample (ru, rv, w, 0)
  DevError* err;
};

constexpr int kGridThreads = 256;
constexpr int kBatch = 64;
// bounded mbarrier waits: a wait gives up after 4 s on the global timer (and
// after 2^26 polls, should the timer not advance)
constexpr unsigned long long kWaitNs = 4000000000ull;
constexpr long long kWaitPolls = 1ll << 26;

struct VisRec {
  int cb;            // footprint origin cell (px0 + P py0) in the padded tile
  int mx, my;        // px0 mod W, py0 mod W
  int w;             // 2S+1 of this CF
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// one-dimensional TMA bulk copy global -> shared, completion on the mbarrier
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// try_wait that may suspend the thread up to hint_ns while the phase is open
__device__ __forceinline__ bool mbar_try_wait_for(unsigned long long* bar, unsigned phase, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait; false when the limit was reached.  The bound is time, not a
// poll count: CTAs of many kernels sharing the SMs (the major-cycle graph runs
// instances side by side) can make an ordinary wait last many polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase) {
  if (mbar_try_wait(bar, phase)) return true;
  const unsigned long long t0 = global_ns();
  for (long long i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait_for(bar, phase, 100000u)) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

__host__ __device__ __forceinline__ unsigned cf_bytes(int w) { return (unsigned)(((w * w * 8) + 15) & ~15); }

// Ring of segment stages shared by the producer warp and the tap warps of
// k_grid and k_degrid_t.  A segment is up to kSeg consecutive sorted samples
// of one run (same tile and CF); its stage holds the CF plane (zero-padded to
// Wp x Wp, brought in by a TMA bulk copy), the samples' records and
// visibilities, and a header {count, index of the segment's first sample in
// the item}.  count < 0 marks the end of the item.
constexpr int kSeg = 32;

__host__ __device__ __forceinline__ int seg_stage_bytes(int cfbuf, int npol) {
  return (cfbuf + kSeg * 16 + kSeg * npol * 8 + 16 + 127) / 128 * 128;
}

// Fewest stages worth keeping two CTAs per SM for: small CF planes come with
// short runs (a segment per sample or so), so the ring must run several
// segments ahead; large ones carry many taps per segment, so two suffice.
static int min_stages_two_ctas(size_t stage) { return stage >= 8192 ? 2 : 4; }

// dynamic shared memory per CTA with three CTAs per SM (228 kB per SM, 1 kB
// reserved per CTA, a little kept for the static variables)
constexpr size_t kSmem3Ctas = 75 * 1024 - 128;

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Producer warp: walks the item's sorted samples 32 at a time (records and
// visibilities loaded one window ahead), cuts each window at CF changes and
// fills one stage per segment.  Returns false when a wait on a stage gave up.
template <int NV>
__device__ __forceinline__ bool seg_produce(const int4 it, const int4* __restrict__ rec,
                                            const float2* __restrict__ vis, int vis_stride, int vis_off,
                                            const float2* __restrict__ cfpad, int Wp2, int cfbuf, int SB, int NST,
                                            unsigned char* ring, unsigned long long* full,
                                            unsigned long long* empty, int& seg, bool stage_cf = true,
                                            const float4* __restrict__ ext = nullptr, int nterm = 1, int pps = 1,
                                            int cfplane = 0, bool cut = true) {
  const int lane = threadIdx.x & 31;
  const unsigned fm = 0xffffffffu;
  const unsigned cfcopy = (unsigned)Wp2 * sizeof(float2);
  seg = 0;
  auto load = [&](int base, int4& r, float2 (&v)[NV > 0 ? NV : 1], float4& x) {
    const int i = base + lane;
    if (i < it.z) {
      r = rec[i];
      if (ext) x = ext[i];
#pragma unroll
      for (int p = 0; p < NV; ++p) v[p] = vis[(size_t)i * vis_stride + vis_off + p];
    } else {
      r = make_int4(0, 0, -1, -1);
    }
  };
  auto acquire = [&](int stage) -> bool {
    bool okw = true;
    if (seg >= NST && lane == 0) okw = mbar_wait(&empty[stage], (unsigned)((seg / NST) - 1) & 1u);
    return __shfl_sync(fm, okw ? 1 : 0, 0) != 0;
  };
  int4 r;
  float2 v[NV > 0 ? NV : 1];
  float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
  load(it.y, r, v, x);
  for (int base = it.y; base < it.z; base += 32) {
    int4 rn;
    float2 vn[NV > 0 ? NV : 1];
    float4 xn = x;
    load(base + 32, rn, vn, xn);                   // next window in flight
    const int nwin = min(32, it.z - base);
    const int zprev = __shfl_up_sync(fm, r.z, 1);
    // segments start at CF changes (cut), else one segment per window
    unsigned heads = __ballot_sync(fm, lane < nwin && (lane == 0 || (cut && zprev != r.z)));
    while (heads) {
      // a stage takes up to pps consecutive runs of the window, each CF plane
      // in a slot of its own; with pps > 1 the staged records carry the slot
      // in place of the CF index
      const int h = __ffs(heads) - 1;
      unsigned rest = heads & (heads - 1);
      int nr = 1;
      while (nr < pps && rest) {
        rest &= rest - 1;
        ++nr;
      }
      const int h2 = rest ? __ffs(rest) - 1 : nwin;
      const unsigned grp = heads & ~rest;
      heads = rest;
      const int stage = seg % NST;
      if (!acquire(stage)) return false;
      unsigned char* sp = ring + (size_t)stage * SB;
      if (lane >= h && lane < h2) {
        int4 rr = r;
        if (pps > 1) rr.z = __popc(grp & (0xffffffffu >> (31 - lane))) - 1;
        reinterpret_cast<int4*>(sp + cfbuf)[lane - h] = rr;
        float2* vs = reinterpret_cast<float2*>(sp + cfbuf + kSeg * 16);
#pragma unroll
        for (int p = 0; p < NV; ++p) vs[(lane - h) * NV + p] = v[p];
        if (ext) reinterpret_cast<float4*>(sp + cfbuf + kSeg * 16 + kSeg * NV * 8)[lane - h] = x;
      }
      if (lane == 0) {
        int* hdr = reinterpret_cast<int*>(sp + SB - 16);
        hdr[0] = h2 - h;
        hdr[1] = base + h - it.y;
      }
      __syncwarp();
      if (stage_cf) {
        if (lane == 0) {
          fence_proxy_async_smem();
          mbar_expect_tx(&full[stage], (unsigned)nr * cfcopy);
        }
        unsigned g = grp;
        for (int k = 0; k < nr; ++k) {
          const int hk = __ffs(g) - 1;
          g &= g - 1;
          const int cfi = __shfl_sync(fm, r.z, hk);
          if (lane == 0) bulk_g2s(sp + (size_t)k * cfplane, cfpad + (size_t)cfi * Wp2, cfcopy, &full[stage]);
        }
      } else if (lane == 0) {
        mbar_arrive(&full[stage]);
      }
      ++seg;
    }
    r = rn;
    x = xn;
#pragma unroll
    for (int p = 0; p < NV; ++p) v[p] = vn[p];
  }
  // end of the item: one terminal segment per consumer that walks its own
  // subsequence of segments (nterm consecutive ones reach every such walk)
  for (int q = 0; q < nterm; ++q) {
    const int stage = seg % NST;
    if (!acquire(stage)) return false;
    if (lane == 0) {
      reinterpret_cast<int*>(ring + (size_t)stage * SB + SB - 16)[0] = -1;
      mbar_arrive(&full[stage]);
    }
    ++seg;
  }
  return true;
}

// After a failed wait: the producer's lane 0 waits (bounded) until the last
// fill of every stage has landed, so no copy is in flight when the CTA exits.
__device__ __forceinline__ void seg_drain(int nfill, int NST, unsigned long long* full) {
  for (int q = 0; q < NST && q < nfill; ++q) {
    const int nq = (nfill - q + NST - 1) / NST;   // fills of stage q
    mbar_wait(&full[q], (unsigned)(nq - 1) & 1u);
  }
}

// Named barrier over the tap warps (the producer warp does not take part).
__device__ __forceinline__ void tap_bar(int nthr) { asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory"); }

// Learned-CF mode: shared memory past the ring's barriers holds the network
// (its shared-memory image, yg_mlp.cuh) and one evaluated CF plane.
__host__ __device__ __forceinline__ size_t learned_smem_bytes(int Wp) {
  return 16 + (size_t)kMlpSmemFloats * sizeof(float) + (size_t)Wp * Wp * sizeof(float2);
}

// The tap warps evaluate CF plane cfi (width w) into `plane` when the segment
// changes CF, between two barriers of their own.
__device__ __forceinline__ void learned_plane(const float* ws, const LearnedCF& L, int cfi, int w, int Wp,
                                              float2* plane, int nthr, int& cur) {
  if (cfi == cur) return;
  tap_bar(nthr);
  // warp-uniform trip counts: every lane of a warp evaluates the network together
  for (int q0 = threadIdx.x & ~31; q0 < Wp * Wp; q0 += nthr) {
    const int q = min(q0 + (int)(threadIdx.x & 31), Wp * Wp - 1);
    const float2 c = mlp_tap_warp(ws, L, cfi, q % Wp, q / Wp, w);
    if (q0 + (int)(threadIdx.x & 31) < Wp * Wp) plane[q] = c;
  }
  tap_bar(nthr);
  cur = cfi;
}

// Continuous learned CF: tap (jx, jy) of a sample with CF index cfi, width w,
// at its own fractional offsets fracu/os + ru, fracv/os + rv and its own w
// (network input xw), instead of the nearest tabulated offset and plane.
// Zero outside the CF width; every lane of the warp calls it together.
__device__ __forceinline__ float2 mlp_tap_exact(const float* __restrict__ ws, const LearnedCF& L, int cfi, int jx,
                                                int jy, int w, const float4& e) {
  const int S = (w - 1) / 2;
  const int fu = cfi % L.os, fv = (cfi / L.os) % L.os;
  const float s1 = 1.f / (float)(S + 1);
  float x[kMlpIn];
  x[0] = ((float)(jx - S) + ((float)fu / (float)L.os + e.x)) * s1;
  x[1] = ((float)(jy - S) + ((float)fv / (float)L.os + e.y)) * s1;
  x[2] = e.z;
  x[3] = 0.f;
  x[4] = 0.f;
  const float2 y = mlp_eval_warp(ws, x);
  if (jx >= w || jy >= w) return make_float2(0.f, 0.f);
  return make_float2(y.x * L.scale, y.y * L.scale);
}

// Gridding of one work item.  Thread/slot k of the tap warps owns the cells
// with (x mod Wp, y mod Wp) = (k mod Wp, k / Wp): no two threads touch the
// same cell, so every tap is accumulated in place in shared memory without
// atomics.  A half-warp holds 16 consecutive residues of one row, so its CF
// taps and grid cells fall on 16 distinct banks (Wp and the CF row stride are
// multiples of 16).  Taps of the padding are exact zeros and land in the
// tile's gutter (columns/rows >= P), which is never read back.
//
// The last warp is the producer: it stages segments (CF plane by TMA, records
// and visibilities by the warp) into an NST-deep ring with full/empty
// mbarriers, so the tap warps read nothing but shared memory and never wait
// on a global load.
//
// CFM selects where the taps come from: 0, the ring (CF plane by TMA); 1, the
// padded CF cache in global memory through L2, for planes too large for the
// ring (the stages then carry records and visibilities only); 2, the learned
// CF: the tap warps evaluate the network for every tap of a new CF plane into
// shared memory when a segment changes CF; 3, the continuous learned CF: every
// tap thread evaluates the network for its own taps of every sample at the
// sample's exact offsets and w (staged beside its record).
//
// RACC (row layouts only): each slot keeps the cell it last accumulated into
// and its running sum in registers, and adds that sum into the shared-memory
// tile only when a sample moves the slot to another cell of its residue class
// (and once at the end of the item), so consecutive samples whose footprints
// cover the slot's cell cost no shared-memory read-modify-write.
template <int NPOL, int MAXSLOTS, int RSTEP, int CFM, bool RACC = false>
__global__ void __launch_bounds__(CFM >= 2 ? 288 : 544) k_grid(GridKArgs a) {
  constexpr bool CFS = CFM == 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nthr = blockDim.x - 32;              // tap threads
  const int ncw = nthr / 32;
  const int Pg = a.Pg;
  const int PG2 = Pg * Pg + nthr;                // per polarisation: tile + one trash cell per tap thread
  float2* acc_s = reinterpret_cast<float2*>(smem_raw);
  unsigned char* ring = smem_raw + (size_t)NPOL * PG2 * sizeof(float2);
  ring = reinterpret_cast<unsigned char*>((reinterpret_cast<size_t>(ring) + 127) & ~(size_t)127);
  const int SB = a.stage_bytes, NST = a.nstages;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(ring + (size_t)NST * SB);
  unsigned long long* empty = full + NST;
  float* ws = reinterpret_cast<float*>((reinterpret_cast<size_t>(empty + NST) + 15) & ~(size_t)15);
  float2* plane = reinterpret_cast<float2*>(ws + kMlpSmemFloats);
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int Wp = a.Wp;
  const int Wp2 = Wp * Wp;
  const int4 it = a.items[blockIdx.x];
  if (CFM >= 2) mlp_load_smem(a.lcf.w16, ws, threadIdx.x, blockDim.x);

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], ncw);
    }
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < NPOL * PG2; i += blockDim.x) acc_s[i] = make_float2(0.f, 0.f);
  __syncthreads();

  int nfill = 0;       // producer: stages filled
  if (warp == ncw) {
    if (!seg_produce<NPOL>(it, a.rec, a.svis, a.npol_total, a.pol0, a.cf.pad, Wp2, a.cfbuf, SB, NST, ring, full,
                           empty, nfill, CFS, CFM == 3 ? a.ext : nullptr, 1, CFS ? a.pps : 1, a.cfplane,
                           CFM != 1)) {
      if (lane == 0) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(1, 1, nfill, blockIdx.x));
        s_abort = 1;
      }
    }
  } else {
    // RSTEP == 0: slot q of thread t owns residue k = q * nthr + t.
    // RSTEP > 0 (nthr = RSTEP * Wp, MAXSLOTS * RSTEP = Wp): thread t owns the
    // x residue t mod Wp and the y residues t / Wp + RSTEP * q, so the x part
    // of the index arithmetic is done once per sample and the slots step down
    // the rows.
    int rx[RSTEP ? 1 : MAXSLOTS], rowoff[RSTEP ? 1 : MAXSLOTS];
    bool live[RSTEP ? 1 : MAXSLOTS];
    if (RSTEP) {
      rx[0] = threadIdx.x % Wp;
      rowoff[0] = threadIdx.x / Wp;
      live[0] = true;
    } else {
#pragma unroll
      for (int q = 0; q < (RSTEP ? 1 : MAXSLOTS); ++q) {
        const int k = q * nthr + threadIdx.x;
        live[q] = k < Wp2;
        rx[q] = live[q] ? k % Wp : 0;
        rowoff[q] = live[q] ? k / Wp : 0;   // ry
      }
    }
    // rows of residues: modulo Wy, the plan's row modulus (the CFs' real width
    // in the exact-rows layout of 16-wide CFs, one slot per thread; Wp otherwise)
    const int Wy = a.Wy;
    const bool rowlive = !RSTEP || rowoff[0] < Wy;
    const int PgR = Pg * RSTEP, WpR = Wp * RSTEP, PgW = Pg * Wy;
    const int trash = Pg * Pg + threadIdx.x;     // target of slots beyond Wp^2
    int cur_cfi = -1;
    // register accumulation: the slot's current cell and its running sums
    int rcell[RACC ? MAXSLOTS : 1];
    float2 racc[RACC ? MAXSLOTS : 1][NPOL];
#pragma unroll
    for (int q = 0; q < (RACC ? MAXSLOTS : 1); ++q) {
      rcell[q] = trash;
#pragma unroll
      for (int p = 0; p < NPOL; ++p) racc[q][p] = make_float2(0.f, 0.f);
    }
    for (int nseg_done = 0;; ++nseg_done) {
      const int stage = nseg_done % NST;
      if (!mbar_wait(&full[stage], (unsigned)(nseg_done / NST) & 1u)) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(1, 2, nseg_done, blockIdx.x));
        s_abort = 1;
        break;
      }
      const unsigned char* sp = ring + (size_t)stage * SB;
      const int cnt = *reinterpret_cast<const volatile int*>(sp + SB - 16);
      if (cnt < 0) break;
      const float2* __restrict__ cf_stage = reinterpret_cast<const float2*>(sp);
      const int4* recs = reinterpret_cast<const int4*>(sp + a.cfbuf);
      const float2* vs = reinterpret_cast<const float2*>(sp + a.cfbuf + kSeg * 16);
      const float4* xs = reinterpret_cast<const float4*>(sp + a.cfbuf + kSeg * 16 + kSeg * NPOL * 8);
      if (CFM == 2) {
        const int4 r0 = recs[0];
        learned_plane(ws, a.lcf, r0.z, (r0.y >> 20) & 0x7ff, Wp, plane, nthr, cur_cfi);
      }
      // register accumulation: the slot's running sums go to the tile when a
      // sample moves the slot to another cell of its residue class
      auto racc_add = [&](const int qq, const int c2, const float2 c, const float2 (&vv)[NPOL]) {
        if (c2 != rcell[qq]) {
          float2 g[NPOL];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) g[p] = acc_s[p * PG2 + rcell[qq]];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            g[p].x += racc[qq][p].x;
            g[p].y += racc[qq][p].y;
            racc[qq][p] = make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int p = 0; p < NPOL; ++p) acc_s[p * PG2 + rcell[qq]] = g[p];
          rcell[qq] = c2;
        }
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          racc[qq][p].x = fmaf(vv[p].x, c.x, fmaf(-vv[p].y, c.y, racc[qq][p].x));
          racc[qq][p].y = fmaf(vv[p].x, c.y, fmaf(vv[p].y, c.x, racc[qq][p].y));
        }
      };
      if (CFM == 1 && RACC && RSTEP != 0) {
        // position-major records (consecutive samples mostly cover the same
        // cells): the taps come through L2, so the taps of a batch of samples
        // are loaded first, all in flight together, then accumulated
        constexpr int PB = MAXSLOTS <= 1 ? 8 : (MAXSLOTS <= 2 ? 4 : 2);
        if (rowlive) {
          for (int l0 = 0; l0 < cnt; l0 += PB) {
            float2 cp[PB][MAXSLOTS];
#pragma unroll
            for (int b = 0; b < PB; ++b) {
              const int4 r = recs[min(l0 + b, cnt - 1)];
              int jx = rx[0] - (r.y & 1023);
              jx += (jx < 0) ? Wp : 0;
              int jy0 = rowoff[0] - ((r.y >> 10) & 1023);
              jy0 += (jy0 < 0) ? Wy : 0;
              const int lim = Wy - jy0;
              const int tap = jx + Wp * jy0;
              const float2* __restrict__ cfp = a.cf.pad + (size_t)r.z * Wp2;
#pragma unroll
              for (int q = 0; q < MAXSLOTS; ++q)
                cp[b][q] = __ldg(cfp + (RSTEP * q >= lim ? tap + WpR * q - Wp * Wy : tap + WpR * q));
            }
#pragma unroll
            for (int b = 0; b < PB; ++b) {
              const int l = l0 + b;
              if (l < cnt) {
                const int4 r = recs[l];
                const bool conj = a.v.pcf && r.y < 0;
                float2 vv[NPOL];
#pragma unroll
                for (int p = 0; p < NPOL; ++p) vv[p] = vs[l * NPOL + p];
                const int cb = (r.x & 0xffff) + Pg * ((r.x >> 16) & 0xffff);
                int jx = rx[0] - (r.y & 1023);
                jx += (jx < 0) ? Wp : 0;
                int jy0 = rowoff[0] - ((r.y >> 10) & 1023);
                jy0 += (jy0 < 0) ? Wy : 0;
                const int lim = Wy - jy0;
                const int cell = cb + jx + Pg * jy0;
#pragma unroll
                for (int q = 0; q < MAXSLOTS; ++q) {
                  const int c2 = RSTEP * q >= lim ? cell + PgR * q - PgW : cell + PgR * q;
                  float2 c = cp[b][q];
                  if (conj) c.y = -c.y;
                  racc_add(RACC ? q : 0, c2, c, vv);
                }
              }
            }
          }
        }
      } else
      for (int l = 0; l < cnt; ++l) {
        const int4 r = recs[l];
        const float2* __restrict__ cf_s =
            CFM == 0 ? (a.pps > 1 ? cf_stage + (size_t)r.z * (a.cfplane / sizeof(float2)) : cf_stage)
                     : (CFM == 1 ? a.cf.pad + (size_t)r.z * Wp2 : plane);
        float4 xe = make_float4(0.f, 0.f, 0.f, 0.f);
        if (CFM == 3) xe = xs[l];
        const int wcf = (r.y >> 20) & 0x7ff;
        const bool conj = a.v.pcf && r.y < 0;   // preconditioner: conjugate CF on this half of the plane
        float2 vv[NPOL];
#pragma unroll
        for (int p = 0; p < NPOL; ++p) vv[p] = vs[l * NPOL + p];
        const int px0 = r.x & 0xffff, py0 = (r.x >> 16) & 0xffff;
        const int cb = px0 + Pg * py0;
        const int mx = r.y & 1023, my = (r.y >> 10) & 1023;
        // continuous learned CF: the taps of every slot, evaluated by the whole
        // warp at once (lanes beyond the residue rows take part and drop theirs)
        float2 ct[CFM == 3 ? MAXSLOTS : 1];
        if (CFM == 3 && RSTEP) {
          int jx = rx[0] - mx;
          jx += (jx < 0) ? Wp : 0;
          int jy0 = rowoff[0] - my;
          jy0 += (jy0 < 0) ? Wy : 0;
          const int lim = Wy - jy0;
#pragma unroll
          for (int q = 0; q < (CFM == 3 ? MAXSLOTS : 1); ++q) {
            const int row = RSTEP * q >= lim ? jy0 + RSTEP * q - Wy : jy0 + RSTEP * q;
            ct[q] = mlp_tap_exact(ws, a.lcf, r.z, jx, row, wcf, xe);
          }
        }
        if (RSTEP && rowlive) {
          int jx = rx[0] - mx;
          jx += (jx < 0) ? Wp : 0;
          int jy0 = rowoff[0] - my;
          jy0 += (jy0 < 0) ? Wy : 0;
          int cell = cb + jx + Pg * jy0;
          int tap = jx + Wp * jy0;
          const int lim = Wy - jy0;     // slots with RSTEP*q >= lim wrap to the top rows
          // taps of the padding hold zeros and are accumulated like the others:
          // predicating them off costs more than it saves.  The network is
          // evaluated only inside the CF width.
#pragma unroll
          for (int q = 0; q < MAXSLOTS; ++q) {
            const bool wrap = RSTEP * q >= lim;
            const int c2 = wrap ? cell - PgW : cell;
            const int t2 = wrap ? tap - Wp * Wy : tap;
            float2 c;
            if (CFM == 3) {
              c = ct[CFM == 3 ? q : 0];
            } else {
              c = CFM == 1 ? __ldg(cf_s + t2) : cf_s[t2];
              if (conj) c.y = -c.y;
            }
            if (RACC) {
              racc_add(RACC ? q : 0, c2, c, vv);
            } else {
              // every polarisation's cell is loaded before any is stored (they are
              // distinct cells), so the loads are in flight together
              float2 g[NPOL];
#pragma unroll
              for (int p = 0; p < NPOL; ++p) g[p] = acc_s[p * PG2 + c2];
#pragma unroll
              for (int p = 0; p < NPOL; ++p) {
                g[p].x = fmaf(vv[p].x, c.x, fmaf(-vv[p].y, c.y, g[p].x));
                g[p].y = fmaf(vv[p].x, c.y, fmaf(vv[p].y, c.x, g[p].y));
              }
#pragma unroll
              for (int p = 0; p < NPOL; ++p) acc_s[p * PG2 + c2] = g[p];
            }
            cell += PgR;
            tap += WpR;
          }
        } else if (!RSTEP) {
#pragma unroll
          for (int q = 0; q < MAXSLOTS; ++q) {
            int jx = rx[q] - mx;
            jx += (jx < 0) ? Wp : 0;
            int jy = rowoff[q] - my;
            jy += (jy < 0) ? Wp : 0;
            const int cell = live[q] ? cb + jx + Pg * jy : trash;
            const int tq = live[q] ? jx + Wp * jy : 0;
            // (the learned CF modes use the row layouts only)
            float2 c = CFM >= 2 ? make_float2(0.f, 0.f) : (CFM == 1 ? __ldg(cf_s + tq) : cf_s[tq]);
            if (CFM < 2 && conj) c.y = -c.y;
            float2 g[NPOL];
#pragma unroll
            for (int p = 0; p < NPOL; ++p) g[p] = acc_s[p * PG2 + cell];
#pragma unroll
            for (int p = 0; p < NPOL; ++p) {
              g[p].x = fmaf(vv[p].x, c.x, fmaf(-vv[p].y, c.y, g[p].x));
              g[p].y = fmaf(vv[p].x, c.y, fmaf(vv[p].y, c.x, g[p].y));
            }
#pragma unroll
            for (int p = 0; p < NPOL; ++p) acc_s[p * PG2 + cell] = g[p];
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[stage]);
    }
    if (RACC) {
      // the running sums of the last cells
#pragma unroll
      for (int q = 0; q < (RACC ? MAXSLOTS : 1); ++q) {
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          float2 g = acc_s[p * PG2 + rcell[q]];
          g.x += racc[q][p].x;
          g.y += racc[q][p].y;
          acc_s[p * PG2 + rcell[q]] = g;
        }
      }
    }
  }
  __syncthreads();
  if (s_abort) {
    if (warp == ncw && lane == 0) seg_drain(nfill, NST, full);
    return;
  }
  const int P = a.P, P2 = P * P;
  float2* out = a.scratch + ((size_t)blockIdx.x * a.npol_total + a.pol0) * P2;
  for (int i = threadIdx.x; i < NPOL * P2; i += blockDim.x) {
    const int p = i / P2, c = i % P2;
    out[i] = acc_s[p * PG2 + (c % P) + Pg * (c / P)];
  }
}

// ---------------------------------------------------------------------------
// k_grid_pl: gridding of one work item whose samples are in plane-major order
// (CF plane, then position in the tile, then oversampling offset), for
// 16-wide CFs with exact residue rows (thread t owns x residue t mod 16 and
// the y residues t / 16 + RY q < Wy of its SL slots, RY = ceil(Wy / SL)).  The producer warp stages records and
// visibilities in segments of up to 32 samples of one CF plane and, when a
// segment starts a new plane, brings every oversampling offset of that plane
// (rows 0..Wy-1 of each padded CF, os^2 bulk copies) into one plane buffer,
// after all earlier segments are consumed.  Consecutive samples of a plane
// mostly cover the same cells, so each thread keeps its cell's running sums
// in registers and adds them into the shared-memory tile only when a sample
// moves it to another cell of its residue class (GridKernel::grid's sums,
// GridKernel.cc:57-97, in another order).
// ---------------------------------------------------------------------------
template <int NPOL, int SL, int NG, bool GT>
__global__ void __launch_bounds__(544) k_grid_pl(GridKArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nthr = blockDim.x - 32;
  const int ncw = nthr / 32;
  const int Pg = a.Pg, Wy = a.Wy, os2 = a.pps;       // pps carries os^2 in this kernel
  const int PG2 = Pg * Pg + nthr;
  // GT: the padded tile lives in this item's scratch slot in global memory
  // (L2), written only by the rare flushes, as reductions; shared memory then
  // holds the plane buffer and the ring only (two CTAs per SM)
  float2* acc_s = GT ? a.scratch + ((size_t)blockIdx.x * a.npol_total + a.pol0) * PG2
                     : reinterpret_cast<float2*>(smem_raw);
  size_t off = GT ? 0 : ((size_t)NPOL * PG2 * sizeof(float2) + 127) & ~(size_t)127;
  float2* planebuf = reinterpret_cast<float2*>(smem_raw + off);
  const int prow = Wy * 16;                           // float2 per oversampling offset
  off += ((size_t)os2 * prow * sizeof(float2) + 127) & ~(size_t)127;
  unsigned char* ring = smem_raw + off;
  const int SB = a.stage_bytes, NST = a.nstages;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(ring + (size_t)NST * SB);
  unsigned long long* empty = full + NST;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int4 it = a.items[blockIdx.x];
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], ncw);
    }
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < NPOL * PG2; i += blockDim.x) acc_s[i] = make_float2(0.f, 0.f);
  __syncthreads();
  int nfill = 0;
  if (warp == ncw) {
    // ---- producer
    const unsigned fm = 0xffffffffu;
    const unsigned rowbytes = (unsigned)prow * sizeof(float2);
    int seg = 0, cur_plane = -1, why = 1;
    bool ok = true;
    const long long ncube = a.v.nrow * (long long)a.v.nchan;
    auto load = [&](int base, int4& r, float2 (&v)[NPOL]) {
      const int i = base + lane;
      if (i < it.z) {
        r = a.rec[i];
        if (a.svis) {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) v[p] = a.svis[(size_t)i * a.npol_total + a.pol0 + p];
        } else {
          // the weighted visibilities straight from the cube (random 8-byte
          // reads, a window ahead of their use, beside a compute-bound kernel)
          const unsigned nr32 = (unsigned)a.v.nrow;
          const int chan = (int)((unsigned)r.w / nr32);
          float pr = 1.f, pi = 0.f;
          if (!a.v.psf && !a.v.pcf) phasor_of(a.v, (long long)((unsigned)r.w - (unsigned)chan * nr32), chan, &pr, &pi);
          const float m = a.v.mfs ? a.v.mfs[chan] : 1.f;
#pragma unroll
          for (int p = 0; p < NPOL; ++p) v[p] = weighted_vis(a.v, r.w, ncube, a.pol0 + p, pr, pi, m);
        }
      } else {
        r = make_int4(0, 0, -1, -1);
      }
    };
    auto acquire = [&](int stage) -> bool {
      bool okw = true;
      if (seg >= NST && lane == 0) okw = mbar_wait(&empty[stage], (unsigned)((seg / NST) - 1) & 1u);
      return __shfl_sync(fm, okw ? 1 : 0, 0) != 0;
    };
    int4 r;
    float2 v[NPOL];
    load(it.y, r, v);
    for (int base = it.y; base < it.z && ok; base += 32) {
      int4 rn;
      float2 vn[NPOL];
      load(base + 32, rn, vn);
      const int nwin = min(32, it.z - base);
      const int pl = r.z >= 0 ? r.z / os2 : -1;
      const int plprev = __shfl_up_sync(fm, pl, 1);
      unsigned heads = __ballot_sync(fm, lane < nwin && (lane == 0 || plprev != pl));
      while (heads) {
        const int h = __ffs(heads) - 1;
        const unsigned rest = heads & (heads - 1);
        const int h2 = rest ? __ffs(rest) - 1 : nwin;
        heads = rest;
        const int stage = seg % NST;
        if (!acquire(stage)) { ok = false; break; }
        unsigned char* sp = ring + (size_t)stage * SB;
        if (lane >= h && lane < h2) {
          // the sample's decode, done once here for every tap thread: footprint
          // origin cell, residues (and the preconditioner's conjugate flag),
          // offset of its oversampling plane in the plane buffer
          const int cb = (r.x & 0xffff) + Pg * ((r.x >> 16) & 0xffff);
          const int res = (r.y & 1023) | (((r.y >> 10) & 1023) << 10) | (r.y & (int)0x80000000);
          reinterpret_cast<int4*>(sp)[lane - h] = make_int4(cb, res, (r.z % os2) * prow, 0);
          float2* vs = reinterpret_cast<float2*>(sp + kSeg * 16);
#pragma unroll
          for (int p = 0; p < NPOL; ++p) vs[(lane - h) * NPOL + p] = v[p];
        }
        const int plane = __shfl_sync(fm, pl, h);
        if (lane == 0) {
          int* hdr = reinterpret_cast<int*>(sp + SB - 16);
          hdr[0] = h2 - h;
        }
        __syncwarp();
        if (plane != cur_plane) {
          // the plane buffer is free once every earlier segment is consumed
          bool okp = true;
          if (lane == 0) {
            if (seg >= 1) okp = mbar_wait(&empty[(seg - 1) % NST], (unsigned)((seg - 1) / NST) & 1u);
            if (okp) {
              fence_proxy_async_smem();
              mbar_expect_tx(&full[stage], (unsigned)os2 * rowbytes);
              for (int f = 0; f < os2; ++f)
                bulk_g2s(planebuf + (size_t)f * prow, a.cf.pad + ((size_t)plane * os2 + f) * 256, rowbytes,
                         &full[stage]);
            }
          }
          if (!__shfl_sync(fm, okp ? 1 : 0, 0)) {
            ok = false;
            why = 3;
            break;
          }
          cur_plane = plane;
        } else if (lane == 0) {
          mbar_arrive(&full[stage]);
        }
        ++seg;
      }
      r = rn;
#pragma unroll
      for (int p = 0; p < NPOL; ++p) v[p] = vn[p];
    }
    if (ok) {
      const int stage = seg % NST;
      if (acquire(stage)) {
        if (lane == 0) {
          reinterpret_cast<int*>(ring + (size_t)stage * SB + SB - 16)[0] = -1;
          mbar_arrive(&full[stage]);
        }
        ++seg;
      } else {
        ok = false;
      }
    }
    nfill = seg;
    if (!ok && lane == 0) {
      raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(2, why, seg, blockIdx.x));
      s_abort = 1;
    }
  } else {
    // ---- tap warps, in NG groups of nthr / NG threads, group g accumulating
    // the polarisations g NPOL / NG ..: thread t of a group owns x residue
    // t mod 16 and the y residues t / 16 + RY q, q < SL (RY = ceil(Wy / SL))
    constexpr int NPG = NPOL / NG;
    const int gsz = nthr / NG;
    const int grp = threadIdx.x / gsz, tl = threadIdx.x - grp * gsz;
    const int pofs = grp * NPG;
    const int RY = (Wy + SL - 1) / SL;
    const int rx = tl & 15, ry0 = tl >> 4;
    int rcell[SL];
    float2 racc[SL][NPG];
#pragma unroll
    for (int q = 0; q < SL; ++q) {
      rcell[q] = Pg * Pg + threadIdx.x;          // this thread's trash cell until the first sample
#pragma unroll
      for (int p = 0; p < NPG; ++p) racc[q][p] = make_float2(0.f, 0.f);
    }
    const bool live = ry0 < RY;
    for (int nseg = 0;; ++nseg) {
      const int stage = nseg % NST;
      if (!mbar_wait(&full[stage], (unsigned)(nseg / NST) & 1u)) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(2, 2, nseg, blockIdx.x));
        s_abort = 1;
        break;
      }
      const unsigned char* sp = ring + (size_t)stage * SB;
      const int cnt = *reinterpret_cast<const volatile int*>(sp + SB - 16);
      if (cnt < 0) break;
      // the staged records, visibilities and CF plane are never written while
      // the tile is: restrict lets the next samples' loads pass this one's stores
      const int4* __restrict__ recs = reinterpret_cast<const int4*>(sp);
      const float2* __restrict__ vs = reinterpret_cast<const float2*>(sp + kSeg * 16);
      const float2* __restrict__ pb = planebuf;
      float2* __restrict__ acc = acc_s;
      if (live) {
#pragma unroll 2
        for (int l = 0; l < cnt; ++l) {
          const int4 r = recs[l];
          const int jx = (rx - (r.y & 1023)) & 15;
          const int my = (r.y >> 10) & 1023;
          const bool conj = a.v.pcf && r.y < 0;
          float2 vv[NPG];
#pragma unroll
          for (int p = 0; p < NPG; ++p) vv[p] = vs[l * NPOL + pofs + p];
#pragma unroll
          for (int q = 0; q < SL; ++q) {
            const int ry = ry0 + RY * q;
            if (SL > 1 && ry >= Wy) continue;
            int jy = ry - my;
            jy += (jy < 0) ? Wy : 0;
            float2 c = pb[r.z + jy * 16 + jx];
            if (conj) c.y = -c.y;
            const int cell = r.x + jx + Pg * jy;
            if (cell != rcell[q]) {
              if (GT) {
                // the thread owns the cell: its reductions land in program order
#pragma unroll
                for (int p = 0; p < NPG; ++p) {
                  float2* gp = acc + (pofs + p) * PG2 + rcell[q];
                  atomicAdd(&gp->x, racc[q][p].x);
                  atomicAdd(&gp->y, racc[q][p].y);
                  racc[q][p] = make_float2(0.f, 0.f);
                }
              } else {
                float2 g[NPG];
#pragma unroll
                for (int p = 0; p < NPG; ++p) g[p] = acc[(pofs + p) * PG2 + rcell[q]];
#pragma unroll
                for (int p = 0; p < NPG; ++p) {
                  g[p].x += racc[q][p].x;
                  g[p].y += racc[q][p].y;
                  racc[q][p] = make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int p = 0; p < NPG; ++p) acc[(pofs + p) * PG2 + rcell[q]] = g[p];
              }
              rcell[q] = cell;
            }
#pragma unroll
            for (int p = 0; p < NPG; ++p) {
              racc[q][p].x = fmaf(vv[p].x, c.x, fmaf(-vv[p].y, c.y, racc[q][p].x));
              racc[q][p].y = fmaf(vv[p].x, c.y, fmaf(vv[p].y, c.x, racc[q][p].y));
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[stage]);
    }
#pragma unroll
    for (int q = 0; q < SL; ++q)
#pragma unroll
      for (int p = 0; p < NPG; ++p) {
        float2* gp = acc_s + (pofs + p) * PG2 + rcell[q];
        if (GT) {
          atomicAdd(&gp->x, racc[q][p].x);
          atomicAdd(&gp->y, racc[q][p].y);
        } else {
          float2 g = *gp;
          g.x += racc[q][p].x;
          g.y += racc[q][p].y;
          *gp = g;
        }
      }
  }
  __syncthreads();
  if (s_abort) {
    if (warp == ncw && lane == 0) seg_drain(nfill, NST, full);
    return;
  }
  if (GT) return;   // the tile is already in the scratch slot
  const int P = a.P, P2 = P * P;
  float2* out = a.scratch + ((size_t)blockIdx.x * a.npol_total + a.pol0) * P2;
  for (int i = threadIdx.x; i < NPOL * P2; i += blockDim.x) {
    const int p = i / P2, c = i % P2;
    out[i] = acc_s[p * PG2 + (c % P) + Pg * (c / P)];
  }
}

// Per sorted sample, once per plan: the footprint origin cell inside the
// padded tile, its residues mod W and the CF width, the CF index, the sample id.
// Bit 31 of the second word marks the half of the uv plane where the
// preconditioner-function gridder uses the conjugate CF
// (TableVisGridder.cc:836-841); other passes ignore it.
__global__ void k_records(const unsigned int* __restrict__ val, const unsigned int* __restrict__ pos,
                          const int* __restrict__ cfi, const unsigned long long* __restrict__ key, long long nvalid,
                          int mbits, int ncf, int kos2, long long ntiles, int ntx, int tile, int smax, int Wp, int Wy,
                          const int* __restrict__ cfsize, int nx, int ny, int4* __restrict__ rec) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid; i += (long long)gridDim.x * blockDim.x) {
    const unsigned int s = val[i];
    const unsigned int ps = pos[s];
    const int c = cfi[s];
    const int w = cfsize[c];
    const int sup = (w - 1) / 2;
    const long long t = key_tile(key[i], mbits, ncf, kos2) % ntiles;
    const int tx = (int)(t % ntx), ty = (int)(t / ntx);
    const int px0 = (int)(ps & 0xffffu) - sup - (tx * tile - smax);
    const int py0 = (int)(ps >> 16) - sup - (ty * tile - smax);
    const int iuo = (int)(ps & 0xffffu), ivo = (int)(ps >> 16);
    const bool conj_half = (ivo < ny / 2 && iuo >= nx / 2) || (ivo <= ny / 2 && iuo < nx / 2);
    rec[i] = make_int4(px0 | (py0 << 16),
                       (int)((unsigned)((px0 % Wp) | ((py0 % Wy) << 10) | (w << 20)) | (conj_half ? 0x80000000u : 0u)),
                       c, (int)s);
  }
}

// Per sorted sample, once per grid pass: the weight checks and
// itsSumWeights(row, pol, image channel) += wt in double (TableVisGridder.cc:
// 783-823) over the sorted records, whose equal sum-of-weights rows come in
// long runs.  Each warp takes chunks of kSumwChunk consecutive samples, 32 at
// a time; a segmented warp scan sums each run of equal rows inside the 32, and
// the run still open at the end of a window is carried into the next window,
// so a run costs one atomic per polarisation per chunk instead of one per 32
// samples (many warps adding into the same few rows at once is what bounds
// this pass).  The sums are exact in FP64 for weights in [1/4, 4], whatever
// the order of the additions.
constexpr int kSumwChunk = 1024;

__global__ void k_sum_weights(VisArgs v, const int4* __restrict__ rec, long long nvalid, SumwArgs sw, DevError* err) {
  const long long n = v.nrow * (long long)v.nchan;
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c0 = warp0 * kSumwChunk; c0 < nvalid; c0 += nwarps * kSumwChunk) {
    const long long c1 = min(nvalid, c0 + kSumwChunk);
    long long cbin = -1;                   // the carried run (same in every lane)
    double cacc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long base = c0; base < c1; base += 32) {
      const long long i = base + lane;
      long long bin = -2;                  // past the chunk: a run of its own, never added
      float wts[4] = {0.f, 0.f, 0.f, 0.f};
      if (i < c1) {
        bin = -1;
        const int4 r = rec[i];
        const long long smp = r.w;
        const unsigned nr32 = (unsigned)v.nrow;     // plans hold fewer than 2^31 samples
        const int chan = (int)((unsigned)r.w / nr32);
        bool good = true;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          if (p >= v.npol) break;
          const float wt = noise_weight(v.noise ? v.noise[smp + n * p].x : 1.f);
          if (!(wt > 0.f)) good = false;
          wts[p] = wt;
        }
        if (!good) raise_error(err, YG_ERR_WEIGHT, smp);
        if (sw.sumw && good) {
          const int rr = sw.track_per_os ? r.z : r.z / (sw.os * sw.os);
          const int ic = sw.chan_map[chan];
          if (rr < 0 || rr >= sw.nrows || ic < 0 || ic >= sw.nchan_img) {
            raise_error(err, YG_ERR_CINDEX, smp);
          } else {
            bin = rr + (long long)sw.nrows * v.npol * ic;
          }
        }
      }
      if (!sw.sumw) continue;              // uniform over the grid: no lane leaves the shuffles
      const long long prev = __shfl_up_sync(full, bin, 1);
      const unsigned heads = __ballot_sync(full, lane == 0 || prev != bin);
      const int seg0 = 31 - __clz(heads & (full >> (31 - lane)));
      const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
      const bool first = seg0 == 0;        // this lane's run starts the window
      const bool last = lane == 31 || (heads >> (lane + 1)) == 0u;   // no run starts after this lane
      const long long bin0 = __shfl_sync(full, bin, 0);
      const bool cont = bin0 == cbin;      // the window's first run continues the carried one
      // the carried run ends here: add it
      if (!cont && cbin >= 0 && lane == 0) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
          if (p < v.npol) atomicAdd(&sw.sumw[cbin + (long long)sw.nrows * p], cacc[p]);
      }
      double lastsum[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        if (p >= v.npol) break;
        double x = bin >= 0 ? (double)wts[p] : 0.0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const double y = __shfl_up_sync(full, x, off);
          if (lane - off >= seg0) x += y;
        }
        if (first && cont) x += cacc[p];
        if (tail && !last && bin >= 0) atomicAdd(&sw.sumw[bin + (long long)sw.nrows * p], x);
        lastsum[p] = __shfl_sync(full, x, 31);
      }
      cbin = __shfl_sync(full, bin, 31);
#pragma unroll
      for (int p = 0; p < 4; ++p) cacc[p] = lastsum[p];
    }
    if (sw.sumw && cbin >= 0 && lane == 0) {
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p < v.npol) atomicAdd(&sw.sumw[cbin + (long long)sw.nrows * p], cacc[p]);
    }
  }
}

// inv[rec[i].w] = i: the sorted index of every on-grid sample (the caller
// sets the others to -1)
__global__ void k_inverse(const int4* __restrict__ rec, long long nvalid, int* __restrict__ inv) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid; i += (long long)gridDim.x * blockDim.x)
    inv[rec[i].w] = (int)i;
}

// The weighted visibilities (weighted_vis), read in the cube's own order
// (sample s = row + nrow * chan, one thread per sample, so each polarisation
// plane is read in coalesced runs) and written to the
// sample's sorted slot inv[s] (its npol values are one contiguous 8 npol-byte
// block).  The weight checks and the sums of weights are k_sum_weights' over
// the sorted records, where equal sum-of-weights rows come in runs.
__global__ void k_gather_cube(VisArgs v, const int* __restrict__ inv, float2* __restrict__ out) {
  const long long n = v.nrow * (long long)v.nchan;
  const unsigned nr32 = (unsigned)v.nrow;       // plans hold fewer than 2^31 samples
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const int i = inv[s];
    if (i < 0) continue;
    const int chan = (int)((unsigned)s / nr32);
    const long long row = (long long)((unsigned)s - (unsigned)chan * nr32);
    float pr = 1.f, pi = 0.f;
    if (!v.psf && !v.pcf) phasor_of(v, row, chan, &pr, &pi);
    const float m = v.mfs ? v.mfs[chan] : 1.f;
    float2 o[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      if (p >= v.npol) break;
      o[p] = weighted_vis(v, s, n, p, pr, pi, m);
    }
    float2* dst = out + (size_t)i * v.npol;
    if (v.npol == 4) {
      reinterpret_cast<float4*>(dst)[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
      reinterpret_cast<float4*>(dst)[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
    } else if (v.npol == 2) {
      reinterpret_cast<float4*>(dst)[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
    } else {
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p < v.npol) dst[p] = o[p];
    }
  }
}

// ---------------------------------------------------------------------------
// k_halo_sum: grid[cell] += sum over items whose padded tile covers the cell.
// One CTA per (grid-plane/channel, tile).  Items of a tile are consecutive.
// ---------------------------------------------------------------------------
struct HaloArgs {
  const int* item_base;      // per tile: first item
  const int* nit;            // per tile: number of items
  const float2* scratch;
  float2* grid;              // ngc planes of (nx, ny, npol) per grid plane
  int nx, ny, npol, nchan_img;
  int tile, ntx, nty;
  long long ntiles;
  int smax, P;
  long long slot_pol;        // scratch elements per polarisation of an item (P^2, or the padded tile)
  int row;                   // scratch row stride (P, or the padded tile's Pg)
};

__global__ void k_halo_sum(HaloArgs a) {
  const long long tid = blockIdx.x;               // over ngc * ntiles
  const long long gc = tid / a.ntiles;
  const long long t = tid % a.ntiles;
  const int tx = (int)(t % a.ntx), ty = (int)(t / a.ntx);
  const int R = (a.smax + a.tile - 1) / a.tile;   // neighbour reach in tiles
  // quick exit when no neighbouring tile holds data
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int q = threadIdx.x; q < (2 * R + 1) * (2 * R + 1); q += blockDim.x) {
    const int ax = tx + q % (2 * R + 1) - R, ay = ty + q / (2 * R + 1) - R;
    if (ax < 0 || ay < 0 || ax >= a.ntx || ay >= a.nty) continue;
    if (a.nit[gc * a.ntiles + ax + (long long)a.ntx * ay] > 0) any = 1;
  }
  __syncthreads();
  if (!any) return;
  const int gind = (int)(gc / a.nchan_img), ichan = (int)(gc % a.nchan_img);
  const long long plane_cells = (long long)a.nx * a.ny;
  const int P2 = a.P * a.P;
  const int T = a.tile;
  for (int c = threadIdx.x; c < T * T * a.npol; c += blockDim.x) {
    const int lx = c % T, ly = (c / T) % T, p = c / (T * T);
    const int x = tx * T + lx, y = ty * T + ly;
    if (x >= a.nx || y >= a.ny) continue;
    float2 sum = make_float2(0.f, 0.f);
    bool hit = false;
    for (int dy = -R; dy <= R; ++dy) {
      const int ay = ty + dy;
      if (ay < 0 || ay >= a.nty) continue;
      const int py = y - (ay * T - a.smax);
      if (py < 0 || py >= a.P) continue;
      for (int dx = -R; dx <= R; ++dx) {
        const int ax = tx + dx;
        if (ax < 0 || ax >= a.ntx) continue;
        const int px = x - (ax * T - a.smax);
        if (px < 0 || px >= a.P) continue;
        const long long nt = gc * a.ntiles + ax + (long long)a.ntx * ay;
        const int m = a.nit[nt];
        if (m == 0) continue;
        const int b = a.item_base[nt];
        for (int j = 0; j < m; ++j) {
          const float2 v = a.scratch[((size_t)(b + j) * a.npol + p) * a.slot_pol + px + (size_t)a.row * py];
          sum.x += v.x;
          sum.y += v.y;
          hit = true;
        }
      }
    }
    if (hit) {
      float2* g = a.grid + (size_t)gind * plane_cells * a.npol * a.nchan_img +
                  plane_cells * (p + (size_t)a.npol * ichan) + x + (size_t)a.nx * y;
      float2 o = *g;
      o.x += sum.x;
      o.y += sum.y;
      *g = o;
    }
  }
}

// ---------------------------------------------------------------------------
// k_degrid: vis = sum CF * conj(grid) (GridKernel.cc:99-137), * mfs, * phasor
// ---------------------------------------------------------------------------
struct DegridKArgs {
  const int4* items;
  const int4* rec;
  const unsigned int* val;
  const unsigned int* pos;
  const int* cfi;
  VisArgs v;
  CFView cf;
  const float2* grid;
  int nx, ny, nchan_img;
  const int* chan_map;
  int tile, ntx;
  long long ntiles;
  int smax, P;
  int smem_grid;             // 1: padded tile staged in shared memory
  float2* out;               // per sample: npol values (sample order)
};

constexpr int kDegridThreads = 256;

// One warp per visibility.  Lanes walk the taps with a shared table of tap ->
// cell offsets and keep four independent partial sums per polarisation so
// that loads of later taps overlap the FMAs of earlier ones; the partial sums
// are combined with warp shuffles.
template <int NPOL>
__global__ void __launch_bounds__(kDegridThreads) k_degrid(DegridKArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int P = a.P, P2 = P * P;
  const int W = 2 * a.smax + 1, W2 = W * W;
  float2* g_s = reinterpret_cast<float2*>(smem_raw);
  int* tab = reinterpret_cast<int*>(smem_raw + (a.smem_grid ? (size_t)NPOL * P2 * sizeof(float2) : 0));
  const int4 it = a.items[blockIdx.x];
  const long long tile_id = it.x;
  const long long gc = tile_id / a.ntiles;
  const long long t = tile_id % a.ntiles;
  const int tx = (int)(t % a.ntx), ty = (int)(t / a.ntx);
  const int X0 = tx * a.tile - a.smax, Y0 = ty * a.tile - a.smax;
  const int gind = (int)(gc / a.nchan_img), ichan = (int)(gc % a.nchan_img);
  const long long plane_cells = (long long)a.nx * a.ny;
  const float2* gbase = a.grid + (size_t)gind * plane_cells * NPOL * a.nchan_img + plane_cells * ((size_t)NPOL * ichan);
  const int stride = a.smem_grid ? P : a.nx;
  for (int i = threadIdx.x; i < W2; i += blockDim.x) tab[i] = (i % W) + stride * (i / W);
  if (a.smem_grid) {
    for (int i = threadIdx.x; i < NPOL * P2; i += blockDim.x) {
      const int px = i % P, py = (i / P) % P, p = i / P2;
      const int x = X0 + px, y = Y0 + py;
      float2 g = make_float2(0.f, 0.f);
      if (x >= 0 && y >= 0 && x < a.nx && y < a.ny) g = gbase[plane_cells * p + x + (size_t)a.nx * y];
      g_s[i] = g;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const float2* src = a.smem_grid ? g_s : gbase;
  const long long pstride = a.smem_grid ? P2 : plane_cells;
  // One sample: the taps of its CF (the reference's loop), then the warp sum
  // and the write-out.  The records are in CF order, so two consecutive
  // samples often share their CF: a warp then takes both at once and each CF
  // tap and offset is loaded once for the two (the same sums in the same order).
  auto finish = [&](const int4 r, float (&re)[4][NPOL], float (&im)[4][NPOL]) {
    const unsigned int s = (unsigned int)r.w;
#pragma unroll
    for (int p = 0; p < NPOL; ++p) {
      float sr = (re[0][p] + re[1][p]) + (re[2][p] + re[3][p]);
      float si = (im[0][p] + im[1][p]) + (im[2][p] + im[3][p]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
      }
      re[0][p] = sr;
      im[0][p] = si;
    }
    if (lane == 0) {
      const long long row = s % a.v.nrow;
      const int chan = (int)(s / a.v.nrow);
      float pr, pi;
      phasor_of(a.v, row, chan, &pr, &pi);
      const float m = a.v.mfs ? a.v.mfs[chan] : 1.f;
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        float cr = re[0][p], ci = im[0][p];
        if (a.v.mfs) { cr = __fmul_rn(cr, m); ci = __fmul_rn(ci, m); }
        const float orr = __fsub_rn(__fmul_rn(cr, pr), __fmul_rn(ci, pi));
        const float oi = __fadd_rn(__fmul_rn(cr, pi), __fmul_rn(ci, pr));
        a.out[(size_t)s * NPOL + p] = make_float2(orr, oi);
      }
    }
  };
  // the footprint origin of a record in the grid source (tile or grid)
  auto origin_of = [&](const int4 r) -> long long {
    const int px0 = r.x & 0xffff, py0 = (r.x >> 16) & 0xffff;
    return a.smem_grid ? (long long)px0 + (long long)P * py0
                       : (long long)(X0 + px0) + (long long)a.nx * (Y0 + py0);
  };
  auto taps_one = [&](const int4 r, float (&re)[4][NPOL], float (&im)[4][NPOL]) {
    const int w = (r.y >> 20) & 1023;
    const long long origin = origin_of(r);
    const float2* __restrict__ cfp = a.cf.data + a.cf.off[r.z];
    const int ntaps = w * w;
    if (w == W) {
      for (int tp = lane; tp < ntaps; tp += 128) {
        int o[4];
        float2 cv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int tu = tp + 32 * u;
          o[u] = tu < ntaps ? tab[tu] : 0;
          cv[u] = tu < ntaps ? __ldg(cfp + tu) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            const float2 g = src[pstride * p + origin + o[u]];
            re[u][p] = fmaf(cv[u].x, g.x, fmaf(cv[u].y, g.y, re[u][p]));
            im[u][p] = fmaf(cv[u].y, g.x, fmaf(-cv[u].x, g.y, im[u][p]));
          }
        }
      }
    } else {
      // plane with its own (smaller) support
      for (int tp = lane; tp < ntaps; tp += 32) {
        const int jx = tp % w, jy = tp / w;
        const float2 cv = __ldg(cfp + tp);
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          const float2 g = src[pstride * p + origin + jx + (long long)stride * jy];
          re[0][p] = fmaf(cv.x, g.x, fmaf(cv.y, g.y, re[0][p]));
          im[0][p] = fmaf(cv.y, g.x, fmaf(-cv.x, g.y, im[0][p]));
        }
      }
    }
  };
  auto zero = [&](float (&re)[4][NPOL], float (&im)[4][NPOL]) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int p = 0; p < NPOL; ++p) { re[u][p] = 0.f; im[u][p] = 0.f; }
  };
  // (pairs for up to two polarisations: four would double 32 accumulators)
  constexpr bool PAIR = NPOL <= 2;
  for (int i = it.y + 2 * warp; i < it.z; i += 2 * nwarps) {
    const int4 r0 = a.rec[i];
    const bool has1 = i + 1 < it.z;
    const int4 r1 = has1 ? a.rec[i + 1] : r0;
    float re[4][NPOL], im[4][NPOL];
    zero(re, im);
    if (PAIR && has1 && r1.z == r0.z && ((r0.y >> 20) & 1023) == W) {
      float re1[4][NPOL], im1[4][NPOL];
      zero(re1, im1);
      const float2* __restrict__ cfp = a.cf.data + a.cf.off[r0.z];
      const long long o0 = origin_of(r0), o1 = origin_of(r1);
      const int ntaps = W2;
      for (int tp = lane; tp < ntaps; tp += 128) {
        int o[4];
        float2 cv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int tu = tp + 32 * u;
          o[u] = tu < ntaps ? tab[tu] : 0;
          cv[u] = tu < ntaps ? __ldg(cfp + tu) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            const float2 g = src[pstride * p + o0 + o[u]];
            const float2 h = src[pstride * p + o1 + o[u]];
            re[u][p] = fmaf(cv[u].x, g.x, fmaf(cv[u].y, g.y, re[u][p]));
            im[u][p] = fmaf(cv[u].y, g.x, fmaf(-cv[u].x, g.y, im[u][p]));
            re1[u][p] = fmaf(cv[u].x, h.x, fmaf(cv[u].y, h.y, re1[u][p]));
            im1[u][p] = fmaf(cv[u].y, h.x, fmaf(-cv[u].x, h.y, im1[u][p]));
          }
        }
      }
      finish(r0, re, im);
      finish(r1, re1, im1);
    } else {
      taps_one(r0, re, im);
      finish(r0, re, im);
      if (has1) {
        zero(re, im);
        taps_one(r1, re, im);
        finish(r1, re, im);
      }
    }
  }
}

// Degridding of one work item on the padded layout: the grid tile (stride Pg,
// zero outside the grid) is staged in shared memory; the producer warp stages
// segments (CF plane by TMA, records) into an NST-deep ring, and tap warp w
// degrids the item's samples whose index in the item is w mod the number of
// tap warps, so the warps work on different segments at once.  A warp walks a
// sample's Wp x Wp taps 32 at a time: a half-warp reads 16 consecutive taps of
// one row, so CF and grid reads fall on distinct banks; padded taps are exact
// zeros.  Four partial sums per lane hide the FMA latency; a warp shuffle
// combines them (GridKernel.cc:99-137).
// Sums V values over the warp with a transposing butterfly: each of the first
// log2(V) exchange steps halves the values a lane carries, the remaining steps
// add one value, so 2V - 1 + 5 - log2(V) shuffles replace 5V.  On return every
// lane holds the warp total of value index lane >> (5 - log2 V).
template <int V>
__device__ __forceinline__ float warp_transpose_sum(float (&x)[V], int lane) {
  static_assert(V == 2 || V == 4 || V == 8, "2, 4 or 8 values");
  int off = 16;
#pragma unroll
  for (int h = V / 2; h >= 1; h /= 2) {
    const bool up = (lane & off) != 0;
#pragma unroll
    for (int k = 0; k < h; ++k) {
      const float send = up ? x[k] : x[k + h];
      const float keep = up ? x[k + h] : x[k];
      x[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
    off >>= 1;
  }
  float y = x[0];
#pragma unroll
  for (; off > 0; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
  return y;
}

struct DegridTArgs {
  const int4* items;
  const int4* rec;
  VisArgs v;
  CFView cf;
  const float2* grid;
  int nx, ny, nchan_img;
  int tile, ntx;
  long long ntiles;
  int smax, Pg, Wp, cfbuf;
  int stage_bytes, nstages;
  int own;                   // segments owned by one warp each (nstages a multiple of the tap warps)
  LearnedCF lcf;             // the network of the learned CF mode
  const float4* ext;         // continuous learned CF: per sorted sample (ru, rv, w, 0)
  float2* out;
  DevError* err;
};

// CFM 0: CF planes by TMA into the ring; 2: the learned CF, evaluated by the
// tap warps into shared memory when a segment changes CF (all tap warps then
// share each segment's samples).
//
// CFM 3: the continuous learned CF, every lane evaluating the network for its
// taps of every sample at the sample's exact offsets and w.
//
// With a.own (not in CFM 2, whose planes the warps evaluate together, and only
// with at least one stage per tap warp), segment s belongs to tap warp
// s mod ncw, which alone waits for it, degrids all its samples and releases
// its stage (empty barriers of count 1).  Otherwise every warp walks every
// segment and takes the samples whose index in the item is its own modulo
// ncw (empty barriers of count ncw).
template <int NPOL, int CFM>
__global__ void __launch_bounds__(288) k_degrid_t(DegridTArgs a) {
  const bool OWN = CFM != 2 && a.own;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int Pg = a.Pg, PG2 = Pg * Pg;
  const int Wp = a.Wp, Wp2 = Wp * Wp;
  float2* g_s = reinterpret_cast<float2*>(smem_raw);
  unsigned char* ring = smem_raw + (size_t)NPOL * PG2 * sizeof(float2);
  ring = reinterpret_cast<unsigned char*>((reinterpret_cast<size_t>(ring) + 127) & ~(size_t)127);
  const int SB = a.stage_bytes, NST = a.nstages;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(ring + (size_t)NST * SB);
  unsigned long long* empty = full + NST;
  float* ws = reinterpret_cast<float*>((reinterpret_cast<size_t>(empty + NST) + 15) & ~(size_t)15);
  float2* plane = reinterpret_cast<float2*>(ws + kMlpSmemFloats);
  __shared__ int s_abort;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int ncw = (blockDim.x >> 5) - 1;
  if (CFM >= 2) mlp_load_smem(a.lcf.w16, ws, threadIdx.x, blockDim.x);

  const int4 it = a.items[blockIdx.x];
  const long long gc = (long long)it.x / a.ntiles;
  const long long t = (long long)it.x % a.ntiles;
  const int tx = (int)(t % a.ntx), ty = (int)(t / a.ntx);
  const int X0 = tx * a.tile - a.smax, Y0 = ty * a.tile - a.smax;
  const int gind = (int)(gc / a.nchan_img), ichan = (int)(gc % a.nchan_img);
  const long long plane_cells = (long long)a.nx * a.ny;
  const float2* gbase = a.grid + (size_t)gind * plane_cells * NPOL * a.nchan_img + plane_cells * ((size_t)NPOL * ichan);

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], OWN ? 1 : ncw);
    }
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < NPOL * PG2; i += blockDim.x) {
    const int p = i / PG2, c = i % PG2;
    const int x = X0 + c % Pg, y = Y0 + c / Pg;
    float2 g = make_float2(0.f, 0.f);
    if (x >= 0 && y >= 0 && x < a.nx && y < a.ny) g = gbase[plane_cells * p + x + (size_t)a.nx * y];
    g_s[i] = g;
  }
  __syncthreads();

  int nfill = 0;
  if (warp == ncw) {
    if (!seg_produce<0>(it, a.rec, nullptr, 0, 0, a.cf.pad, Wp2, a.cfbuf, SB, NST, ring, full, empty, nfill,
                        CFM == 0, CFM == 3 ? a.ext : nullptr, OWN ? ncw : 1)) {
      if (lane == 0) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(3, 1, nfill, blockIdx.x));
        s_abort = 1;
      }
    }
  } else {
    // lane's first tap and its grid-cell offset inside the footprint
    const int jx0 = lane % Wp, jy0 = lane / Wp;
    const int steps = Wp2 / 32;        // Wp is a multiple of 16: Wp^2 / 32 is a multiple of 8
    const int rows_per_step = 32 / Wp; // 2 when Wp == 16, else 0 (wrap handled below)
    int cur_cfi = -1;
    for (int nseg = OWN ? warp : 0;; nseg += OWN ? ncw : 1) {
      const int stage = nseg % NST;
      if (!mbar_wait(&full[stage], (unsigned)(nseg / NST) & 1u)) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(3, 2, nseg, blockIdx.x));
        s_abort = 1;
        break;
      }
      const unsigned char* sp = ring + (size_t)stage * SB;
      const volatile int* hdr = reinterpret_cast<const volatile int*>(sp + SB - 16);
      const int cnt = hdr[0];
      if (cnt < 0) break;
      const int g0 = hdr[1];
      const float2* __restrict__ cf_s = CFM == 2 ? plane : reinterpret_cast<const float2*>(sp);
      const int4* recs = reinterpret_cast<const int4*>(sp + a.cfbuf);
      const float4* xs = reinterpret_cast<const float4*>(sp + a.cfbuf + kSeg * 16);
      if (CFM == 2) {
        const int4 r0 = recs[0];
        learned_plane(ws, a.lcf, r0.z, (r0.y >> 20) & 0x7ff, Wp, plane, 32 * ncw, cur_cfi);
      }
      for (int l = OWN ? 0 : (CFM == 2 ? warp : (warp - g0 % ncw + ncw) % ncw); l < cnt; l += OWN ? 1 : ncw) {
        const int4 r = recs[l];
        float4 xe = make_float4(0.f, 0.f, 0.f, 0.f);
        if (CFM == 3) xe = xs[l];
        const int wcf = (r.y >> 20) & 0x7ff;
        const int px0 = r.x & 0xffff, py0 = (r.x >> 16) & 0xffff;
        const int origin = px0 + Pg * py0;
        float re[4][NPOL], im[4][NPOL];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int p = 0; p < NPOL; ++p) re[u][p] = im[u][p] = 0.f;
        int tap = lane;
        int jx = jx0;
        int row = jy0;
        int cell = origin + jx0 + Pg * jy0;
        // one step of 32 taps into partial sum u
        auto step = [&](const int u) {
          // taps of the padding hold zeros in the table (read unconditionally,
          // which keeps the four partial sums' loads independent); the
          // network is evaluated only inside the CF width
          const float2 cv = CFM == 3 ? mlp_tap_exact(ws, a.lcf, r.z, jx, row, wcf, xe) : cf_s[tap];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            const float2 g = g_s[p * PG2 + cell];
            re[u][p] = fmaf(cv.x, g.x, fmaf(cv.y, g.y, re[u][p]));
            im[u][p] = fmaf(cv.y, g.x, fmaf(-cv.x, g.y, im[u][p]));
          }
          tap += 32;
          if (rows_per_step) {
            cell += rows_per_step * Pg;
            row += rows_per_step;
          } else {
            jx += 32;
            const bool wrap = jx >= Wp;
            jx = wrap ? jx - Wp : jx;
            row += wrap ? 1 : 0;
            cell += wrap ? 32 - Wp + Pg : 32;
          }
        };
        // rows at and below the CF width hold only zero taps: the steps stop at
        // the last one that reaches a row inside it (7 of 8 for 13-wide CFs in
        // 16-wide planes); step st always feeds partial sum st mod 4
        const int nst = min(steps, (wcf * Wp + 31) >> 5);
        int st = 0;
        for (; st + 4 <= nst; st += 4) {
#pragma unroll
          for (int u = 0; u < 4; ++u) step(u);
        }
#pragma unroll
        for (int u = 0; u < 3; ++u)
          if (st + u < nst) step(u);
        // values 2p (real) and 2p + 1 (imaginary) of polarisation p
        float x[2 * NPOL];
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          x[2 * p] = (re[0][p] + re[1][p]) + (re[2][p] + re[3][p]);
          x[2 * p + 1] = (im[0][p] + im[1][p]) + (im[2][p] + im[3][p]);
        }
        constexpr int sh = NPOL == 4 ? 2 : (NPOL == 2 ? 3 : 4);   // 5 - log2(2 NPOL)
        const float cr0 = warp_transpose_sum<2 * NPOL>(x, lane);
        const float ci0 = __shfl_down_sync(0xffffffffu, cr0, 1 << sh);
        const int v = lane >> sh;
        if ((lane & ((1 << sh) - 1)) == 0 && (v & 1) == 0) {
          const int p = v >> 1;
          const long long s = r.w;
          // row and channel only for the phasor and the MFS weight (sample
          // ids and row counts of a plan are below 2^31: 32-bit division)
          float pr = 1.f, pi = 0.f;
          int chan = 0;
          if (a.v.delay || a.v.mfs) {
            const unsigned su = (unsigned)r.w, nr = (unsigned)a.v.nrow;
            chan = (int)(su / nr);
            phasor_of(a.v, (long long)(su - (unsigned)chan * nr), chan, &pr, &pi);
          }
          float cr = cr0, ci = ci0;
          if (a.v.mfs) {
            const float m = a.v.mfs[chan];
            cr = __fmul_rn(cr, m);
            ci = __fmul_rn(ci, m);
          }
          a.out[(size_t)s * NPOL + p] = make_float2(__fsub_rn(__fmul_rn(cr, pr), __fmul_rn(ci, pi)),
                                                    __fadd_rn(__fmul_rn(cr, pi), __fmul_rn(ci, pr)));
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[stage]);
    }
  }
  __syncthreads();
  if (s_abort && warp == ncw && lane == 0) seg_drain(nfill, NST, full);
}

// Sum of V values per lane over the 16 lanes of each half-warp, transposed
// as in warp_transpose_sum: value v of a half ends in its lanes with
// (lane & 15) >> (4 - log2 V) == v.
template <int V>
__device__ __forceinline__ float half_transpose_sum(float (&x)[V], int lane) {
  static_assert(V == 2 || V == 4 || V == 8 || V == 16, "2, 4, 8 or 16 values");
  int off = 8;
#pragma unroll
  for (int h = V / 2; h >= 1; h /= 2) {
    const bool up = (lane & off) != 0;
#pragma unroll
    for (int k = 0; k < h; ++k) {
      const float send = up ? x[k] : x[k + h];
      const float keep = up ? x[k + h] : x[k];
      x[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
    off >>= 1;
  }
  float y = x[0];
#pragma unroll
  for (; off > 0; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
  return y;
}

// GridKernel::degrid (GridKernel.cc:99-137) for 16-wide CF planes without the
// learned CF: k_degrid_t's item, tile and segment ring, with the tap warps
// working differently.  Warp s mod ncw degrids segment s (one CF plane, up to
// kSeg samples); with a.own it alone waits for and releases the segment (the
// ring protocol of k_degrid_t's owned segments), otherwise every tap warp
// waits for every segment and releases it, passing over the others' (empty
// barriers of count ncw, one terminal segment).  A warp takes its segment's
// samples two at a time, one per half-warp: lane jx = lane & 15 of a half walks the rows of its sample's
// footprint (one 16-wide grid row per half-warp load, which is one
// shared-memory wavefront per 64-bit load), and keeps the column jx of the
// segment's CF plane, rows 0..w-1, in registers, read once per segment rather
// than once per sample and tap.  Rows past the CF width w are not visited.
// SPH = 2: each half-warp takes two samples at a time (four per warp pass),
// whose independent sums keep twice the loads in flight.
template <int NPOL, int SPH>
__global__ void __launch_bounds__(288) k_degrid_r(DegridTArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int Wp = 16;
  const int Pg = a.Pg, PG2 = Pg * Pg;
  float2* g_s = reinterpret_cast<float2*>(smem_raw);
  unsigned char* ring = smem_raw + (size_t)NPOL * PG2 * sizeof(float2);
  ring = reinterpret_cast<unsigned char*>((reinterpret_cast<size_t>(ring) + 127) & ~(size_t)127);
  const int SB = a.stage_bytes, NST = a.nstages;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(ring + (size_t)NST * SB);
  unsigned long long* empty = full + NST;
  __shared__ int s_abort;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int ncw = (blockDim.x >> 5) - 1;

  const int4 it = a.items[blockIdx.x];
  const long long gc = (long long)it.x / a.ntiles;
  const long long t = (long long)it.x % a.ntiles;
  const int tx = (int)(t % a.ntx), ty = (int)(t / a.ntx);
  const int X0 = tx * a.tile - a.smax, Y0 = ty * a.tile - a.smax;
  const int gind = (int)(gc / a.nchan_img), ichan = (int)(gc % a.nchan_img);
  const long long plane_cells = (long long)a.nx * a.ny;
  const float2* gbase = a.grid + (size_t)gind * plane_cells * NPOL * a.nchan_img + plane_cells * ((size_t)NPOL * ichan);

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], a.own ? 1 : ncw);
    }
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < NPOL * PG2; i += blockDim.x) {
    const int p = i / PG2, c = i % PG2;
    const int x = X0 + c % Pg, y = Y0 + c / Pg;
    float2 g = make_float2(0.f, 0.f);
    if (x >= 0 && y >= 0 && x < a.nx && y < a.ny) g = gbase[plane_cells * p + x + (size_t)a.nx * y];
    g_s[i] = g;
  }
  __syncthreads();

  int nfill = 0;
  if (warp == ncw) {
    if (!seg_produce<0>(it, a.rec, nullptr, 0, 0, a.cf.pad, Wp * Wp, a.cfbuf, SB, NST, ring, full, empty, nfill,
                        true, nullptr, a.own ? ncw : 1)) {
      if (lane == 0) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(4, 1, nfill, blockIdx.x));
        s_abort = 1;
      }
    }
  } else {
    const int jx = lane & 15, half = lane >> 4;
    constexpr int V = 2 * NPOL * SPH;
    constexpr int sh = V == 16 ? 0 : (V == 8 ? 1 : (V == 4 ? 2 : 3));   // 4 - log2(V)
    for (int nseg = a.own ? warp : 0;; nseg += a.own ? ncw : 1) {
      const int stage = nseg % NST;
      if (!mbar_wait(&full[stage], (unsigned)(nseg / NST) & 1u)) {
        raise_error(a.err, YG_ERR_TIMEOUT, timeout_where(4, 2, nseg, blockIdx.x));
        s_abort = 1;
        break;
      }
      const unsigned char* sp = ring + (size_t)stage * SB;
      const volatile int* hdr = reinterpret_cast<const volatile int*>(sp + SB - 16);
      const int cnt = hdr[0];
      if (cnt < 0) break;
      if (!a.own && nseg % ncw != warp) {
        // another warp's segment: pass it
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        continue;
      }
      const float2* __restrict__ cf_s = reinterpret_cast<const float2*>(sp);
      const int4* recs = reinterpret_cast<const int4*>(sp + a.cfbuf);
      // the segment's CF width and this lane's CF column
      const int w = min(Wp, (recs[0].y >> 20) & 0x7ff);
      float2 cv[Wp];
#pragma unroll
      for (int k = 0; k < Wp; ++k) cv[k] = k < w ? cf_s[k * Wp + jx] : make_float2(0.f, 0.f);
      for (int l = 0; l < cnt; l += 2 * SPH) {
        // sample u of this half: l + half + 2 u
        int4 rr[SPH];
        int origin[SPH];
#pragma unroll
        for (int u = 0; u < SPH; ++u) {
          const int li = l + half + 2 * u;
          rr[u] = recs[li < cnt ? li : l];
          origin[u] = (rr[u].x & 0xffff) + Pg * ((rr[u].x >> 16) & 0xffff) + jx;
        }
        // SPH == 1: two partial sums (even and odd rows) for independent chains
        constexpr int NPART = SPH == 1 ? 2 : 1;
        float re[SPH][NPART][NPOL], im[SPH][NPART][NPOL];
#pragma unroll
        for (int u = 0; u < SPH; ++u)
#pragma unroll
          for (int q = 0; q < NPART; ++q)
#pragma unroll
            for (int p = 0; p < NPOL; ++p) re[u][q][p] = im[u][q][p] = 0.f;
#pragma unroll
        for (int k = 0; k < Wp; ++k) {
          if (k < w) {
            const float2 c = cv[k];
            constexpr int Q = 0;
#pragma unroll
            for (int u = 0; u < SPH; ++u) {
              const int cell = origin[u] + Pg * k;
              const int q = NPART == 2 ? (k & 1) : Q;
#pragma unroll
              for (int p = 0; p < NPOL; ++p) {
                const float2 g = g_s[p * PG2 + cell];
                re[u][q][p] = fmaf(c.x, g.x, fmaf(c.y, g.y, re[u][q][p]));
                im[u][q][p] = fmaf(c.y, g.x, fmaf(-c.x, g.y, im[u][q][p]));
              }
            }
          }
        }
        float x[V];
#pragma unroll
        for (int u = 0; u < SPH; ++u)
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            x[2 * NPOL * u + 2 * p] = NPART == 2 ? re[u][0][p] + re[u][NPART - 1][p] : re[u][0][p];
            x[2 * NPOL * u + 2 * p + 1] = NPART == 2 ? im[u][0][p] + im[u][NPART - 1][p] : im[u][0][p];
          }
        const float cr0 = half_transpose_sum<V>(x, lane);
        const float ci0 = __shfl_down_sync(0xffffffffu, cr0, 1 << sh);
        const int v = (lane & 15) >> sh;
        const int u = v / (2 * NPOL);
        const bool mine = l + half + 2 * u < cnt;
        if (mine && (lane & ((1 << sh) - 1)) == 0 && (v & 1) == 0) {
          const int4 r = u == 0 ? rr[0] : rr[SPH - 1];
          const int p = (v % (2 * NPOL)) >> 1;
          float pr = 1.f, pi = 0.f;
          int chan = 0;
          if (a.v.delay || a.v.mfs) {
            const unsigned su = (unsigned)r.w, nr = (unsigned)a.v.nrow;
            chan = (int)(su / nr);
            phasor_of(a.v, (long long)(su - (unsigned)chan * nr), chan, &pr, &pi);
          }
          float cr = cr0, ci = ci0;
          if (a.v.mfs) {
            const float m = a.v.mfs[chan];
            cr = __fmul_rn(cr, m);
            ci = __fmul_rn(ci, m);
          }
          a.out[(size_t)r.w * NPOL + p] = make_float2(__fsub_rn(__fmul_rn(cr, pr), __fmul_rn(ci, pi)),
                                                      __fadd_rn(__fmul_rn(cr, pi), __fmul_rn(ci, pr)));
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[stage]);
    }
  }
  __syncthreads();
  if (s_abort && warp == ncw && lane == 0) seg_drain(nfill, NST, full);
}

// shared memory of k_degrid_t: the grid tile per polarisation, then the ring
static size_t degrid_t_tile_bytes(int npol, int Pg) { return (size_t)npol * Pg * Pg * sizeof(float2) + 128; }

size_t degrid_t_smem_bytes(int npol, int Pg, int cfbuf, int nst) {
  return degrid_t_tile_bytes(npol, Pg) + (size_t)nst * (seg_stage_bytes(cfbuf, 0) + 16);
}

// Ring depth of k_degrid_t and k_degrid_r: up to 16 stages (two per tap
// warp), as many as fit with two CTAs per SM when at
// least min_stages_two_ctas do, else as many as fit one CTA; 0 when not even 2
// fit.
int degrid_t_stages(int npol, int Pg, int cfbuf) {
  const size_t tile = degrid_t_tile_bytes(npol, Pg);
  const size_t stage = (size_t)seg_stage_bytes(cfbuf, 0) + 16;
  // three CTAs per SM when a stage per tap warp fits beside the tile (small tiles)
  if (tile + 8 * stage <= kSmem3Ctas) return (int)std::min<size_t>(16, (kSmem3Ctas - tile) / stage);
  if (tile + min_stages_two_ctas(stage) * stage <= 113 * 1024)
    return (int)std::min<size_t>(16, (113 * 1024 - tile) / stage);
  if (tile + 2 * stage <= 227 * 1024) return (int)std::min<size_t>(16, (227 * 1024 - tile) / stage);
  return 0;
}

// prev[o] = o when sample (row, chan) with o = row * nchan + chan is on-grid,
// -1 otherwise (input of the max-scan)
__global__ void k_order_marks(const unsigned char* __restrict__ status, long long nrow, int nchan, int want,
                              int* __restrict__ marks) {
  const long long n = nrow * (long long)nchan;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long row = o / nchan;
    const int chan = (int)(o % nchan);
    const long long s = row + nrow * chan;
    marks[o] = (status[s] >= want) ? (int)o : -1;
  }
}

// vis(row, chan, pol) += value; off-grid valid samples receive the value of the
// most recent on-grid sample in the reference's loop order (row outer, channel
// inner), or the value carried over from the previous call.
__global__ void k_degrid_writeback(const unsigned char* __restrict__ status, const int* __restrict__ prev,
                                   const float2* __restrict__ vals, const float2* __restrict__ carry,
                                   long long nrow, int nchan, int npol, float2* __restrict__ vis) {
  // sample order s = row + nrow * chan: the cube's own order, so the
  // read-modify-write of vis and the reads of vals are coalesced; only
  // off-grid samples (status 2) look up their loop-order predecessor
  const long long n = nrow * (long long)nchan;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const unsigned char st = status[s];
    if (st < 2) continue;
    long long src = s;
    if (st != 3) {
      const long long o = (s % nrow) * nchan + s / nrow;
      const int q = prev[o];
      src = q >= 0 ? (q / nchan) + nrow * (q % nchan) : -1;
    }
    for (int p = 0; p < npol; ++p) {
      const float2 v = src >= 0 ? vals[(size_t)src * npol + p] : carry[p];
      float2 o2 = vis[s + n * p];
      o2.x += v.x;
      o2.y += v.y;
      vis[s + n * p] = o2;
    }
  }
}

// *last = the largest loop-order index o = row * nchan + chan whose sample has
// status >= want (stays -1 when there is none); *last must be -1 on entry
__global__ void k_last_marked(const unsigned char* __restrict__ status, long long nrow, int nchan, int want,
                              int* __restrict__ last) {
  const long long n = nrow * (long long)nchan;
  int best = -1;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    if (status[s] >= want) best = max(best, (int)((s % nrow) * nchan + s / nrow));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0 && best >= 0) atomicMax(last, best);
}

// carry_out = value of the sample with loop-order index *q (unchanged if q < 0)
__global__ void k_update_carry(const int* __restrict__ qp, long long nrow, int nchan, int npol,
                               const float2* __restrict__ vals, int vals_are_vis, float2* __restrict__ carry) {
  const long long n = nrow * (long long)nchan;
  if (n == 0) return;
  const int q = *qp;
  if (q < 0) return;
  const long long sq = (q / nchan) + nrow * (q % nchan);
  for (int p = threadIdx.x; p < npol; p += blockDim.x) {
    carry[p] = vals_are_vis ? vals[sq + n * p] : vals[(size_t)sq * npol + p];
  }
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
static inline int grid_dim(long long n, int threads, int cap = 148 * 32) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

static int ceil_log2(unsigned long long v) {
  int b = 0;
  while ((1ull << b) < v && b < 63) ++b;
  return b;
}

#define YG_CUDA_TRY(x)                          \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return YG_ERR_CUDA;  \
  } while (0)

// Position-major key of sorted sample i: (grid plane and tile, Morton
// position in the tile, CF index), from its CF-major key (grid plane and tile,
// CF index, Morton position); the value is i.
// mode 2, plane-major: (grid plane and tile, CF plane = CF index / os^2,
// Morton position, oversampling offset = CF index mod os^2).
__global__ void k_pos_keys(const unsigned long long* __restrict__ key, long long nvalid, int mbits, int ncf,
                           int mode, int os2, unsigned long long* __restrict__ key2, unsigned int* __restrict__ idx) {
  const unsigned long long mmask = (1ull << mbits) - 1ull;
  const unsigned long long ncp = (unsigned long long)(ncf / os2);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = key[i];
    const unsigned long long hi = k >> mbits;
    const unsigned long long gct = hi / (unsigned long long)ncf, cfi = hi % (unsigned long long)ncf;
    if (mode == 2) {
      const unsigned long long cp = cfi / (unsigned long long)os2, fr = cfi % (unsigned long long)os2;
      key2[i] = (((((gct * ncp + cp) << mbits) | (k & mmask)) * (unsigned long long)os2) + fr);
    } else {
      key2[i] = (((gct << mbits) | (k & mmask)) * (unsigned long long)ncf) + cfi;
    }
    idx[i] = (unsigned int)i;
  }
}

__global__ void k_permute_rec(const int4* __restrict__ rec, const unsigned int* __restrict__ perm, long long n,
                              int4* __restrict__ out) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
    out[j] = rec[perm[j]];
}

// out[0] = work items (base of the last tile + its item count), out[1] = on-grid samples
__global__ void k_plan_counts(const int* __restrict__ last_base, const int* __restrict__ last_n,
                              const long long* __restrict__ nvalid, long long* out) {
  out[0] = (long long)*last_base + *last_n;
  out[1] = *nvalid;
}

// Bins one chunk: fills plan (sorted ids, tile table, work items).
int plan_build(Plan& pl, const BinArgs& a, int vmax, DevError* err, cudaStream_t st) {
  const long long n = a.nrow * (long long)a.nchan;
  pl.nsamples = n;
  pl.wy = a.wy > 0 ? a.wy : a.cf.wpad;
  pl.prev_ready = false;
  pl.ext_ready = false;
  pl.mbits = a.mbits;
  pl.ncf = a.cf.ncf;
  pl.nrow = a.nrow;
  pl.nchan = a.nchan;
  pl.npol = a.npol;
  pl.tile = a.tile;
  pl.ntx = a.ntx;
  pl.nty = a.nty;
  pl.vmax = vmax;
  pl.smax = (a.cf.maxsize - 1) / 2;
  pl.pad = a.tile + 2 * pl.smax;
  int ngrid_planes = 1;
  if (a.grid_mode == GRID_MODE_WPLANE) ngrid_planes = a.ws.nwplanes;
  if (a.grid_mode == GRID_MODE_STACK) ngrid_planes = a.ws_stack.nwplanes;
  pl.ngc = ngrid_planes * a.nchan_img;
  pl.ntiles_total = (long long)pl.ngc * a.ntx * a.nty;
  if (n == 0) {
    pl.nvalid = 0;
    pl.nitems = 0;
    return YG_OK;
  }
  if (n >= (1ll << 31)) return YG_ERR_ARG;  // sort sizes and tile offsets are int
  YG_CUDA_TRY(pl.key.ensure(n * 8));
  YG_CUDA_TRY(pl.key_alt.ensure(n * 8));
  YG_CUDA_TRY(pl.val.ensure(n * 4));
  YG_CUDA_TRY(pl.val_alt.ensure(n * 4));
  YG_CUDA_TRY(pl.pos.ensure(n * 4));
  YG_CUDA_TRY(pl.cfi.ensure(n * 4));
  YG_CUDA_TRY(pl.status.ensure(n));
  k_bin<<<grid_dim(n, 256), 256, 0, st>>>(a, pl.key.as<unsigned long long>(), pl.val.as<unsigned int>(),
                                          pl.pos.as<unsigned int>(), pl.cfi.as<int>(),
                                          pl.status.as<unsigned char>(), err);
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(cudaGetLastError());
  // radix sort over the bits that keys use (the invalid key is one past the
  // largest valid key, so it sorts last)
  const int end_bit = std::min(64, ceil_log2(a.invalid_key + 1));
  YG_CUDA_TRY(pl.sort_tmp.ensure(std::max(sort_pairs_tmp_bytes(n), scan_tmp_bytes(n))));
  int in_alt = 0;
  YG_CUDA_TRY(sort_pairs(pl.key.as<unsigned long long>(), pl.key_alt.as<unsigned long long>(),
                         pl.val.as<unsigned int>(), pl.val_alt.as<unsigned int>(), n, end_bit, pl.sort_tmp.p,
                         pl.sort_tmp.bytes, st, &in_alt));
  if (in_alt) {
    std::swap(pl.key.p, pl.key_alt.p);
    std::swap(pl.key.bytes, pl.key_alt.bytes);
    std::swap(pl.val.p, pl.val_alt.p);
    std::swap(pl.val.bytes, pl.val_alt.bytes);
  }
  // tile table
  const long long nt = pl.ntiles_total;
  YG_CUDA_TRY(pl.tstart.ensure(nt * 4));
  YG_CUDA_TRY(pl.tend.ensure(nt * 4));
  YG_CUDA_TRY(pl.nit.ensure(nt * 4));
  YG_CUDA_TRY(pl.itembase.ensure((nt + 1) * 4));
  YG_CUDA_TRY(pl.nvalid_d.ensure(16));
  YG_CUDA_TRY(cudaMemsetAsync(pl.tstart.p, 0, nt * 4, st));
  YG_CUDA_TRY(cudaMemsetAsync(pl.tend.p, 0, nt * 4, st));
  YG_CUDA_TRY(cudaMemsetAsync(pl.nvalid_d.p, 0, 16, st));
  const int kos2 = a.key_planes ? a.os * a.os : 1;
  k_tile_bounds<<<grid_dim(n, 256), 256, 0, st>>>(pl.key.as<unsigned long long>(), n, a.mbits, a.cf.ncf, kos2,
                                                  a.invalid_key, pl.tstart.as<int>(), pl.tend.as<int>(),
                                                  pl.nvalid_d.as<long long>());
  YG_COUNT_LAUNCH();
  k_count_items<<<grid_dim(nt, 256), 256, 0, st>>>(pl.tstart.as<int>(), pl.tend.as<int>(), nt, vmax, pl.nit.as<int>());
  YG_COUNT_LAUNCH();
  if (scan_tmp_bytes(nt) > pl.sort_tmp.bytes) YG_CUDA_TRY(pl.sort_tmp.ensure(scan_tmp_bytes(nt)));
  YG_CUDA_TRY(scan_i32(pl.nit.as<int>(), pl.itembase.as<int>(), nt, SCAN_SUM, true, pl.sort_tmp.p, pl.sort_tmp.bytes,
                       st));
  // item count and on-grid samples back to the host through mapped memory
  YG_CUDA_TRY(pl.info_h.ensure(16));
  k_plan_counts<<<1, 1, 0, st>>>(pl.itembase.as<int>() + (nt - 1), pl.nit.as<int>() + (nt - 1),
                                 pl.nvalid_d.as<long long>(), pl.info_h.as<long long>());
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(cudaStreamSynchronize(st));
  pl.nitems = (int)pl.info_h.as<volatile long long>()[0];
  pl.nvalid = pl.info_h.as<volatile long long>()[1];
  YG_CUDA_TRY(pl.items.ensure_headroom((size_t)std::max(1, pl.nitems) * sizeof(int4)));
  k_fill_items<<<grid_dim(nt, 256), 256, 0, st>>>(pl.tstart.as<int>(), pl.tend.as<int>(), pl.nit.as<int>(),
                                                  pl.itembase.as<int>(), nt, vmax, pl.items.as<int4>());
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(pl.rec.ensure_headroom((size_t)std::max(1ll, pl.nvalid) * sizeof(int4)));
  if (pl.nvalid > 0) {
    if (a.cf.wpad > 1023 || !a.cf.pad) return YG_ERR_UNSUPPORTED;  // residues are packed in 10 bits
    k_records<<<grid_dim(pl.nvalid, 256), 256, 0, st>>>(pl.val.as<unsigned int>(), pl.pos.as<unsigned int>(),
                                                        pl.cfi.as<int>(), pl.key.as<unsigned long long>(), pl.nvalid,
                                                        a.mbits, a.cf.ncf, kos2, (long long)a.ntx * a.nty, a.ntx, a.tile,
                                                        pl.smax, a.cf.wpad, pl.wy, a.cf.size, a.nx, a.ny,
                                                        pl.rec.as<int4>());
    YG_COUNT_LAUNCH();
  }
  pl.inv_ready = pl.inv_pos_ready = false;
  if (a.need_inv && !a.key_planes) {
    YG_CUDA_TRY(pl.inv.ensure((size_t)n * 4));
    YG_CUDA_TRY(cudaMemsetAsync(pl.inv.p, 0xff, (size_t)n * 4, st));
    if (pl.nvalid > 0) {
      k_inverse<<<grid_dim(pl.nvalid, 256), 256, 0, st>>>(pl.rec.as<int4>(), pl.nvalid, pl.inv.as<int>());
      YG_COUNT_LAUNCH();
    }
    pl.inv_ready = true;
  }
  pl.pos_ready = false;
  pl.grid_only = false;
  if (a.key_planes) {
    // a gridding-only plan sorted once by the plane-major key: its records
    // are the plane-major order itself (no CF-major records, no second sort)
    std::swap(pl.rec.p, pl.rec_pos.p);
    std::swap(pl.rec.bytes, pl.rec_pos.bytes);
    pl.grid_only = true;
    pl.pos_ready = pl.nvalid > 0;
    pl.pos_mode = 2;
    pl.os2 = a.os * a.os;
  } else if (a.pos_major && pl.nvalid > 0) {
    // a second order of the same records for gridding: tile first as before
    // (the work items stay valid), then the position inside the tile, then
    // the CF index, so consecutive samples of an item mostly cover the same
    // cells (register accumulation in k_grid)
    const long long nv = pl.nvalid;
    // key_alt and val_alt (free once the records are made) hold the new
    // keys; the primary keys, read last by k_pos_keys, are the sort's
    // alternate key buffer; only the alternate values need a buffer of
    // their own (the primary values stay in use by the passes)
    YG_CUDA_TRY(pl.pos_val2.ensure_headroom(nv * 4));
    k_pos_keys<<<grid_dim(nv, 256), 256, 0, st>>>(pl.key.as<unsigned long long>(), nv, a.mbits, a.cf.ncf,
                                                  a.pos_major, a.os * a.os, pl.key_alt.as<unsigned long long>(),
                                                  pl.val_alt.as<unsigned int>());
    YG_COUNT_LAUNCH();
    if (sort_pairs_tmp_bytes(nv) > pl.sort_tmp.bytes) YG_CUDA_TRY(pl.sort_tmp.ensure(sort_pairs_tmp_bytes(nv)));
    int alt2 = 0;
    YG_CUDA_TRY(sort_pairs(pl.key_alt.as<unsigned long long>(), pl.key.as<unsigned long long>(),
                           pl.val_alt.as<unsigned int>(), pl.pos_val2.as<unsigned int>(), nv, end_bit,
                           pl.sort_tmp.p, pl.sort_tmp.bytes, st, &alt2));
    YG_CUDA_TRY(pl.rec_pos.ensure_headroom((size_t)nv * sizeof(int4)));
    k_permute_rec<<<grid_dim(nv, 256), 256, 0, st>>>(pl.rec.as<int4>(),
                                                     alt2 ? pl.pos_val2.as<unsigned int>() : pl.val_alt.as<unsigned int>(),
                                                     nv, pl.rec_pos.as<int4>());
    YG_COUNT_LAUNCH();
    if (a.pos_major == 1) {
      // the position-major kernel reads gathered visibilities in this order
      YG_CUDA_TRY(pl.inv_pos.ensure((size_t)n * 4));
      YG_CUDA_TRY(cudaMemsetAsync(pl.inv_pos.p, 0xff, (size_t)n * 4, st));
      k_inverse<<<grid_dim(nv, 256), 256, 0, st>>>(pl.rec_pos.as<int4>(), nv, pl.inv_pos.as<int>());
      YG_COUNT_LAUNCH();
      pl.inv_pos_ready = true;
    }
    YG_CUDA_TRY(cudaGetLastError());
    pl.pos_ready = true;
    pl.pos_mode = a.pos_major;
    pl.os2 = a.os * a.os;
  }
  YG_CUDA_TRY(cudaGetLastError());
  return YG_OK;
}


template <int NPOL, int MAXSLOTS, int RSTEP, int CFM = 0, bool RACC = false>
static cudaError_t launch_grid_ms(const GridKArgs& g, int nitems, int threads, size_t smem, cudaStream_t st) {
  auto k = k_grid<NPOL, MAXSLOTS, RSTEP, CFM, RACC>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<nitems, threads + 32, smem, st>>>(g);   // tap warps + the producer warp
  YG_COUNT_LAUNCH();
  return cudaGetLastError();
}

// threads x slots covering Wp^2 residue classes: the row layout where one
// exists for Wp, else the least-waste generic layout (threads a multiple of
// 32, at most 512)
struct GridShape {
  int threads, slots, rstep;
};

GridShape grid_shape(int Wp);

// Row layouts with fewer tap threads and more slots per thread, selected by
// the tuning variant: variant v > 1 divides the threads of the default row
// layout by 2^(v-1) (each thread then steps down 2^(v-1) times as many rows).
GridShape grid_shape_variant(int Wp, int variant) {
  GridShape sh = grid_shape(Wp);
  if (variant <= 1 || sh.rstep == 0) return sh;
  for (int v = 1; v < variant; ++v) {
    if (sh.rstep % 2 || sh.threads / 2 < 64 || (sh.threads / 2) % 32) return GridShape{0, 0, 0};
    sh = GridShape{sh.threads / 2, sh.slots * 2, sh.rstep / 2};
  }
  return sh;
}

GridShape grid_shape(int Wp) {
  switch (Wp) {
    case 16: return GridShape{256, 1, 16};
    case 32: return GridShape{256, 4, 8};
    case 48: return GridShape{384, 6, 8};
    case 64: return GridShape{512, 8, 8};
    case 80: return GridShape{320, 20, 4};
    case 96: return GridShape{384, 24, 4};
    case 112: return GridShape{448, 28, 4};
    case 128: return GridShape{512, 32, 4};
    case 144: return GridShape{288, 72, 2};
    default: break;
  }
  const int W2 = Wp * Wp;
  const int cand[10] = {1, 2, 3, 4, 6, 8, 9, 12, 16, 25};
  GridShape best{0, 0, 0};
  long long best_waste = -1;
  for (int sl : cand) {
    int th = ((W2 + sl - 1) / sl + 31) / 32 * 32;
    if (th < 64) th = 64;
    if (th > 512) continue;
    const long long waste = (long long)th * sl - W2;
    if (best_waste < 0 || waste < best_waste || (waste == best_waste && th > best.threads)) {
      best = GridShape{th, sl, 0};
      best_waste = waste;
    }
  }
  return best;
}

// CF taps from global memory: the row layouts of the widest CFs only
template <int NPOL>
static cudaError_t launch_grid_np_global(const GridKArgs& g, int nitems, size_t smem, GridShape sh,
                                         cudaStream_t st) {
  const int t = sh.threads;
  switch (sh.slots * 1000 + sh.rstep) {
    case 8008: return launch_grid_ms<NPOL, 8, 8, 1>(g, nitems, t, smem, st);
    case 20004: return launch_grid_ms<NPOL, 20, 4, 1>(g, nitems, t, smem, st);
    case 24004: return launch_grid_ms<NPOL, 24, 4, 1>(g, nitems, t, smem, st);
    case 28004: return launch_grid_ms<NPOL, 28, 4, 1>(g, nitems, t, smem, st);
    case 32004: return launch_grid_ms<NPOL, 32, 4, 1>(g, nitems, t, smem, st);
    case 72002: return launch_grid_ms<NPOL, 72, 2, 1>(g, nitems, t, smem, st);
    default: return cudaErrorInvalidConfiguration;
  }
}

// learned CF: the row layouts of at most 256 tap threads (register budget of
// the in-kernel network)
GridShape grid_shape_learned(int Wp) {
  switch (Wp) {
    case 16: return GridShape{256, 1, 16};
    case 32: return GridShape{256, 4, 8};
    case 48: return GridShape{192, 12, 4};
    case 64: return GridShape{256, 16, 4};
    default: return GridShape{0, 0, 0};
  }
}

template <int NPOL>
static cudaError_t launch_grid_np_learned(const GridKArgs& g, int nitems, size_t smem, GridShape sh,
                                          cudaStream_t st) {
  const int t = sh.threads;
  switch (sh.slots * 1000 + sh.rstep) {
    case 1016: return g.ext ? launch_grid_ms<NPOL, 1, 16, 3>(g, nitems, t, smem, st)
                            : launch_grid_ms<NPOL, 1, 16, 2>(g, nitems, t, smem, st);
    case 4008: return g.ext ? launch_grid_ms<NPOL, 4, 8, 3>(g, nitems, t, smem, st)
                            : launch_grid_ms<NPOL, 4, 8, 2>(g, nitems, t, smem, st);
    case 12004: return g.ext ? launch_grid_ms<NPOL, 12, 4, 3>(g, nitems, t, smem, st)
                             : launch_grid_ms<NPOL, 12, 4, 2>(g, nitems, t, smem, st);
    case 16004: return g.ext ? launch_grid_ms<NPOL, 16, 4, 3>(g, nitems, t, smem, st)
                             : launch_grid_ms<NPOL, 16, 4, 2>(g, nitems, t, smem, st);
    default: return cudaErrorInvalidConfiguration;
  }
}

template <int NPOL>
static cudaError_t launch_grid_np(const GridKArgs& g, int nitems, size_t smem, GridShape sh, cudaStream_t st,
                                  bool racc = false) {
  const int t = sh.threads;
  if (g.pos_major) {
    // position-major records, taps through L2, register accumulation (row layouts only)
    if (!sh.rstep) return cudaErrorInvalidConfiguration;
    switch (sh.slots * 1000 + sh.rstep) {
      case 1016: return launch_grid_ms<NPOL, 1, 16, 1, true>(g, nitems, t, smem, st);
      case 2008: return launch_grid_ms<NPOL, 2, 8, 1, true>(g, nitems, t, smem, st);
      case 4008: return launch_grid_ms<NPOL, 4, 8, 1, true>(g, nitems, t, smem, st);
      case 6008: return launch_grid_ms<NPOL, 6, 8, 1, true>(g, nitems, t, smem, st);
      case 8008: return launch_grid_ms<NPOL, 8, 8, 1, true>(g, nitems, t, smem, st);
      default: return cudaErrorInvalidConfiguration;
    }
  }
  if (sh.rstep && racc) {
    // register accumulation: layouts of at most 8 slots per thread
    switch (sh.slots * 1000 + sh.rstep) {
      case 1016: return launch_grid_ms<NPOL, 1, 16, 0, true>(g, nitems, t, smem, st);
      case 2008: return launch_grid_ms<NPOL, 2, 8, 0, true>(g, nitems, t, smem, st);
      case 4004: return launch_grid_ms<NPOL, 4, 4, 0, true>(g, nitems, t, smem, st);
      case 4008: return launch_grid_ms<NPOL, 4, 8, 0, true>(g, nitems, t, smem, st);
      case 6008: return launch_grid_ms<NPOL, 6, 8, 0, true>(g, nitems, t, smem, st);
      case 8004: return launch_grid_ms<NPOL, 8, 4, 0, true>(g, nitems, t, smem, st);
      case 8008: return launch_grid_ms<NPOL, 8, 8, 0, true>(g, nitems, t, smem, st);
      default: break;   // wider layouts accumulate in shared memory
    }
  }
  if (sh.rstep) {
    switch (sh.slots * 1000 + sh.rstep) {
      case 1016: return launch_grid_ms<NPOL, 1, 16>(g, nitems, t, smem, st);
      case 2008: return launch_grid_ms<NPOL, 2, 8>(g, nitems, t, smem, st);
      case 4004: return launch_grid_ms<NPOL, 4, 4>(g, nitems, t, smem, st);
      case 8004: return launch_grid_ms<NPOL, 8, 4>(g, nitems, t, smem, st);
      case 12004: return launch_grid_ms<NPOL, 12, 4>(g, nitems, t, smem, st);
      case 16004: return launch_grid_ms<NPOL, 16, 4>(g, nitems, t, smem, st);
      case 8002: return launch_grid_ms<NPOL, 8, 2>(g, nitems, t, smem, st);
      case 4008: return launch_grid_ms<NPOL, 4, 8>(g, nitems, t, smem, st);
      case 6008: return launch_grid_ms<NPOL, 6, 8>(g, nitems, t, smem, st);
      case 8008: return launch_grid_ms<NPOL, 8, 8>(g, nitems, t, smem, st);
      case 20004: return launch_grid_ms<NPOL, 20, 4>(g, nitems, t, smem, st);
      case 24004: return launch_grid_ms<NPOL, 24, 4>(g, nitems, t, smem, st);
      case 28004: return launch_grid_ms<NPOL, 28, 4>(g, nitems, t, smem, st);
      case 32004: return launch_grid_ms<NPOL, 32, 4>(g, nitems, t, smem, st);
      case 72002: return launch_grid_ms<NPOL, 72, 2>(g, nitems, t, smem, st);
      default: return cudaErrorInvalidConfiguration;
    }
  }
  switch (sh.slots) {
    case 1: return launch_grid_ms<NPOL, 1, 0>(g, nitems, t, smem, st);
    case 2: return launch_grid_ms<NPOL, 2, 0>(g, nitems, t, smem, st);
    case 3: return launch_grid_ms<NPOL, 3, 0>(g, nitems, t, smem, st);
    case 4: return launch_grid_ms<NPOL, 4, 0>(g, nitems, t, smem, st);
    case 6: return launch_grid_ms<NPOL, 6, 0>(g, nitems, t, smem, st);
    case 8: return launch_grid_ms<NPOL, 8, 0>(g, nitems, t, smem, st);
    case 9: return launch_grid_ms<NPOL, 9, 0>(g, nitems, t, smem, st);
    case 12: return launch_grid_ms<NPOL, 12, 0>(g, nitems, t, smem, st);
    case 16: return launch_grid_ms<NPOL, 16, 0>(g, nitems, t, smem, st);
    case 25: return launch_grid_ms<NPOL, 25, 0>(g, nitems, t, smem, st);
    default: break;
  }
  return cudaErrorInvalidConfiguration;
}

// shared memory of k_grid: the guttered tile (Pg^2 + one trash cell per tap
// thread) per polarisation, then the ring of segment stages and its 2 NST
// mbarriers
int grid_cf_buffer_bytes(int wpad) { return ((wpad * wpad * 8) + 127) / 128 * 128; }

int grid_tile_stride(int tile, int wpad, int smax, bool varsup) { return tile + wpad - 1 + (varsup ? smax : 0); }

static size_t grid_tile_bytes(int npol, int Pg, int nthr) {
  return (size_t)npol * ((size_t)Pg * Pg + nthr) * sizeof(float2) + 128;
}

size_t grid_smem_bytes(int npol, int Pg, int cfbuf, int nthr, int nst) {
  return grid_tile_bytes(npol, Pg, nthr) + (size_t)nst * (seg_stage_bytes(cfbuf, npol) + 16);
}

// Ring depth: up to 8 stages, as many as fit with two CTAs per SM when at
// least min_stages_two_ctas do, else as many as fit one CTA; 0 when not even 2
// fit.
int grid_stages(int npol, int Pg, int cfbuf, int nthr) {
  const size_t tile = grid_tile_bytes(npol, Pg, nthr);
  const size_t stage = (size_t)seg_stage_bytes(cfbuf, npol) + 16;
  // three CTAs per SM when the tile is small enough to leave room for the stages
  if (tile + std::max(3, min_stages_two_ctas(stage)) * stage <= kSmem3Ctas)
    return (int)std::min<size_t>(8, (kSmem3Ctas - tile) / stage);
  if (tile + min_stages_two_ctas(stage) * stage <= 113 * 1024)
    return (int)std::min<size_t>(8, (113 * 1024 - tile) / stage);
  if (tile + 2 * stage <= 227 * 1024) return (int)std::min<size_t>(8, (227 * 1024 - tile) / stage);
  return 0;
}

// Tile side for a plan: the largest multiple of 8 (32..256) whose k_grid
// tile leaves room for min_stages_two_ctas segment stages with two CTAs per
// SM, else for 3 stages with one CTA per SM, for the polarisations of one pass.
int grid_tile_for(int smax, int npol, bool varsup) {
  const int wpad = ((2 * smax + 1) + 15) / 16 * 16;
  const int cfbuf = (wpad <= 16 ? 4 : 1) * grid_cf_buffer_bytes(wpad);   // the stage's CF slots (see plan_grid)
  const GridShape sh = grid_shape(wpad);
  if (sh.threads == 0) return 16;
  const size_t budgets[2] = {113 * 1024, 227 * 1024};
  for (int k = 0; k < 2; ++k) {
    for (int npa : {npol, 2, 1}) {
      if (npa > npol || npol % npa) continue;
      const size_t stage = (size_t)seg_stage_bytes(cfbuf, npa) + 16;
      const int nst = k == 0 ? min_stages_two_ctas(stage) : 3;
      for (int t = 256; t >= 32; t -= 8) {
        const int Pg = grid_tile_stride(t, wpad, smax, varsup);
        if (grid_tile_bytes(npa, Pg, sh.threads) + nst * stage <= budgets[k]) return t;
      }
    }
  }
  // CF planes read from global memory: stages of records only, one CTA per SM
  const size_t stage = (size_t)seg_stage_bytes(0, 1) + 16;
  for (int t = 256; t >= 8; t -= 8) {
    const int Pg = grid_tile_stride(t, wpad, smax, varsup);
    if (grid_tile_bytes(1, Pg, sh.threads) + 4 * stage <= budgets[1]) return t;
  }
  return 8;
}

// Polarisations accumulated together in one k_grid pass: the most that fit
// the shared-memory budget.
int grid_pols_per_pass(int npol, int Pg, int cfbuf, int nthr) {
  const int cands[3] = {4, 2, 1};
  for (int c : cands) {
    if (c > npol || npol % c) continue;
    if (grid_stages(c, Pg, cfbuf, nthr) > 0) return c;
  }
  return 0;
}

// Grids the samples of a plan onto `grid` (ngrid planes of (nx, ny, npol, nchan_img)).
int plan_grid(const Plan& pl, const VisArgs& v, const CFView& cf, float2* grid, int nx, int ny, int nchan_img,
              const SumwArgs& sw, DevBuf& scratch, DevBuf& svis, DevError* err, cudaStream_t st, cudaEvent_t ev0,
              cudaEvent_t ev1, int mode, const LearnedCF* lcf) {
  const bool learned = lcf && lcf->w16;
  // mode bits: 16 register accumulation of the row layouts; 32 the
  // position-major records with taps read through L2 (and register accumulation)
  // mode 64: the plane-major records with each CF plane's offsets staged in
  // shared memory (k_grid_pl: 16-wide CFs in exact residue rows)
  const bool planes = (mode & 64) != 0 && pl.pos_ready && pl.pos_mode == 2 && !learned && cf.wpad == 16 &&
                      pl.wy > 0 && pl.wy <= 16 && !cf.varsup && v.npol <= 4;
  const bool pos = !planes && (mode & 32) != 0 && pl.pos_ready && pl.pos_mode == 1 && !learned && v.npol <= 4;
  const bool racc = (mode & 16) != 0 || pos;
  if (pl.grid_only && !planes && pl.nitems > 0) return YG_ERR_STATE;   // only the plane-major kernel reads it
  // mode 128 (with 64): the plane-major kernel's tile in the item's scratch slot
  const bool gtile = planes && (mode & 128) != 0;
  mode &= 15;
  // plane-major kernel layout: 1 one residue row per thread; 2 the same in two
  // groups of threads, each accumulating half the polarisations; 3 two rows per thread
  const int pl_sl = mode == 3 ? 2 : 1;
  const int pl_ng = (mode == 2 && v.npol >= 2) ? 2 : 1;
  const int gtile_nthr = planes ? pl_ng * ((16 * ((pl.wy + pl_sl - 1) / pl_sl) + 31) / 32 * 32) : 0;
  if (learned && v.pcf) return YG_ERR_UNSUPPORTED;
  if (pl.nitems == 0) return YG_OK;
  if (!cf.pad || cf.wpad <= 0) return YG_ERR_STATE;
  const int P = pl.pad;
  const int Pg = grid_tile_stride(pl.tile, cf.wpad, pl.smax, cf.varsup != 0);
  GridShape shape = learned ? grid_shape_learned(cf.wpad) : grid_shape_variant(cf.wpad, mode);
  if (pl.wy != cf.wpad) {
    // exact rows: thread t owns x residue t mod 16 and y residue t / 16 < wy
    if (cf.wpad != 16 || pl.wy > 16 || (!learned && mode > 1 && !planes)) return YG_ERR_UNSUPPORTED;
    shape = GridShape{(16 * pl.wy + 31) / 32 * 32, 1, 16};
  }
  if (shape.threads == 0) return YG_ERR_UNSUPPORTED;
  const size_t per_item = gtile ? (size_t)v.npol * ((size_t)Pg * Pg + gtile_nthr) * sizeof(float2)
                                : (size_t)v.npol * P * P * sizeof(float2);
  YG_CUDA_TRY(scratch.ensure_headroom(per_item * pl.nitems));
  if (v.npol > 4) return YG_ERR_UNSUPPORTED;
  // the weighted visibilities in the order of the records the kernel reads,
  // gathered in the cube's order (the plane-major kernel's producer forms its
  // own); the weight checks and the sums of weights over the sorted records
  if (!planes) {
    if (!(pos ? pl.inv_pos_ready : pl.inv_ready)) return YG_ERR_STATE;   // a plan made for degridding only
    YG_CUDA_TRY(svis.ensure_headroom((size_t)std::max(1ll, pl.nvalid) * v.npol * sizeof(float2)));
    k_gather_cube<<<grid_dim(pl.nsamples, 256), 256, 0, st>>>(v, pos ? pl.inv_pos.as<int>() : pl.inv.as<int>(),
                                                             svis.as<float2>());
    YG_COUNT_LAUNCH();
  }
  k_sum_weights<<<grid_dim(pl.nvalid, 256), 256, 0, st>>>(v, planes ? pl.rec_pos.as<int4>() : pl.rec.as<int4>(),
                                                          pl.nvalid, sw, err);
  YG_COUNT_LAUNCH();
  GridKArgs g;
  g.Wy = pl.wy;
  g.pos_major = pos ? 1 : 0;
  g.items = pl.items.as<int4>();
  g.val = pl.val.as<unsigned int>();
  g.rec = pos ? pl.rec_pos.as<int4>() : pl.rec.as<int4>();
  g.svis = planes ? nullptr : svis.as<float2>();
  g.pos = pl.pos.as<unsigned int>();
  g.cfi = pl.cfi.as<int>();
  g.v = v;
  g.cf = cf;
  g.tile = pl.tile;
  g.ntx = pl.ntx;
  g.ntiles = (long long)pl.ntx * pl.nty;
  g.smax = pl.smax;
  g.P = P;
  g.Pg = Pg;
  g.Wp = cf.wpad;
  g.cfplane = grid_cf_buffer_bytes(cf.wpad);
  // small planes come with short runs: several runs share a stage
  g.pps = (!learned && cf.wpad <= 16) ? 4 : 1;
  g.cfbuf = g.pps * g.cfplane;
  g.scratch = scratch.as<float2>();
  g.npol_total = v.npol;
  g.err = err;
  // the last warp is the producer: the tap threads must fill whole warps
  if (shape.threads % 32) return YG_ERR_UNSUPPORTED;
  g.lcf = learned ? *lcf : LearnedCF{};
  g.ext = learned ? lcf->ext : nullptr;
  const int xv = g.ext ? 2 : 0;          // the continuous inputs take two float2 slots per sample
  int npa;
  bool cf_global = false;
  size_t smem;
  if (learned) {
    // records-only stages, then the network and one evaluated CF plane
    g.cfbuf = 0;
    const size_t extra = learned_smem_bytes(cf.wpad);
    npa = 0;
    for (int c : {4, 2, 1}) {
      if (c > v.npol || v.npol % c) continue;
      const size_t st_c = (size_t)seg_stage_bytes(0, c + xv) + 16;
      if (grid_tile_bytes(c, Pg, shape.threads) + extra + 2 * st_c <= 227 * 1024) { npa = c; break; }
    }
    if (npa == 0) return YG_ERR_UNSUPPORTED;
    const size_t st_n = (size_t)seg_stage_bytes(0, npa + xv) + 16;
    const size_t tile_b = grid_tile_bytes(npa, Pg, shape.threads);
    g.nstages = (int)std::min<size_t>(8, (227 * 1024 - tile_b - extra) / st_n);
    g.stage_bytes = seg_stage_bytes(0, npa + xv);
    smem = tile_b + (size_t)g.nstages * st_n + extra;
  } else {
    npa = pos ? 0 : grid_pols_per_pass(v.npol, Pg, g.cfbuf, shape.threads);
    cf_global = npa == 0;      // CF planes too wide for the ring (or position-major records): taps from global memory
    if (cf_global) {
      g.cfbuf = 0;
      npa = grid_pols_per_pass(v.npol, Pg, 0, shape.threads);
      if (npa == 0) return YG_ERR_UNSUPPORTED;
    }
    g.nstages = grid_stages(npa, Pg, g.cfbuf, shape.threads);
    g.stage_bytes = seg_stage_bytes(g.cfbuf, npa);
    smem = grid_smem_bytes(npa, Pg, g.cfbuf, shape.threads, g.nstages);
  }
  if (planes) {
    // k_grid_pl: tile + one plane of every oversampling offset + the ring
    const int os2 = pl.os2;
    const int sl = pl_sl, ng = pl_ng, nthr_pl = gtile_nthr;
    const size_t plane_b = ((size_t)os2 * pl.wy * 16 * sizeof(float2) + 127) & ~(size_t)127;
    g.rec = pl.rec_pos.as<int4>();
    g.pps = os2;
    g.cfbuf = 0;
    npa = 0;
    for (int c : {4, 2, 1}) {
      if (c > v.npol || v.npol % c) continue;
      const size_t tile_b =
          gtile ? 0 : ((size_t)c * ((size_t)Pg * Pg + nthr_pl) * sizeof(float2) + 127) & ~(size_t)127;
      const size_t stage = (size_t)seg_stage_bytes(0, c) + 16;
      // two CTAs per SM where the tile is in global memory and the plane fits twice
      const size_t budget = (gtile && plane_b + 2 * stage + 256 <= 113 * 1024) ? 113 * 1024 - 256 : 227 * 1024;
      if (tile_b + plane_b + 2 * stage <= budget) {
        npa = c;
        g.nstages = (int)std::min<size_t>(8, (budget - tile_b - plane_b) / stage);
        g.stage_bytes = seg_stage_bytes(0, c);
        smem = tile_b + plane_b + (size_t)g.nstages * stage;
        break;
      }
    }
    if (npa == 0) return YG_ERR_UNSUPPORTED;
    if (ev0) cudaEventRecord(ev0, st);
    for (int pol0 = 0; pol0 < v.npol; pol0 += npa) {
      g.pol0 = pol0;
      auto launch = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<pl.nitems, nthr_pl + 32, smem, st>>>(g);
        YG_COUNT_LAUNCH();
      };
      const int ngl = npa >= 2 ? ng : 1;
      if (ngl != ng) return YG_ERR_UNSUPPORTED;
      switch (npa * 100 + sl * 10 + ngl + (gtile ? 1000 : 0)) {
        case 111: launch(k_grid_pl<1, 1, 1, false>); break;
        case 121: launch(k_grid_pl<1, 2, 1, false>); break;
        case 211: launch(k_grid_pl<2, 1, 1, false>); break;
        case 212: launch(k_grid_pl<2, 1, 2, false>); break;
        case 221: launch(k_grid_pl<2, 2, 1, false>); break;
        case 411: launch(k_grid_pl<4, 1, 1, false>); break;
        case 412: launch(k_grid_pl<4, 1, 2, false>); break;
        case 421: launch(k_grid_pl<4, 2, 1, false>); break;
        case 1111: launch(k_grid_pl<1, 1, 1, true>); break;
        case 1211: launch(k_grid_pl<2, 1, 1, true>); break;
        case 1212: launch(k_grid_pl<2, 1, 2, true>); break;
        case 1411: launch(k_grid_pl<4, 1, 1, true>); break;
        case 1412: launch(k_grid_pl<4, 1, 2, true>); break;
        default: return YG_ERR_UNSUPPORTED;
      }
      YG_CUDA_TRY(cudaGetLastError());
    }
  } else {
  if (ev0) cudaEventRecord(ev0, st);
  for (int pol0 = 0; pol0 < v.npol; pol0 += npa) {
    g.pol0 = pol0;
    cudaError_t e;
    if (learned) {
      switch (npa) {
        case 1: e = launch_grid_np_learned<1>(g, pl.nitems, smem, shape, st); break;
        case 2: e = launch_grid_np_learned<2>(g, pl.nitems, smem, shape, st); break;
        default: e = launch_grid_np_learned<4>(g, pl.nitems, smem, shape, st); break;
      }
      if (e == cudaErrorInvalidConfiguration) return YG_ERR_UNSUPPORTED;
      if (e != cudaSuccess) return YG_ERR_CUDA;
      continue;
    }
    switch (npa * 2 + (cf_global ? 1 : 0)) {
      case 2: e = launch_grid_np<1>(g, pl.nitems, smem, shape, st, racc); break;
      case 4: e = launch_grid_np<2>(g, pl.nitems, smem, shape, st, racc); break;
      case 8: e = launch_grid_np<4>(g, pl.nitems, smem, shape, st, racc); break;
      case 3: e = pos ? launch_grid_np<1>(g, pl.nitems, smem, shape, st, true)
                      : launch_grid_np_global<1>(g, pl.nitems, smem, shape, st); break;
      case 5: e = pos ? launch_grid_np<2>(g, pl.nitems, smem, shape, st, true)
                      : launch_grid_np_global<2>(g, pl.nitems, smem, shape, st); break;
      case 9: e = pos ? launch_grid_np<4>(g, pl.nitems, smem, shape, st, true)
                      : launch_grid_np_global<4>(g, pl.nitems, smem, shape, st); break;
      default: return YG_ERR_UNSUPPORTED;
    }
    if (e == cudaErrorInvalidConfiguration) return YG_ERR_UNSUPPORTED;
    if (e != cudaSuccess) return YG_ERR_CUDA;
  }
  }
  if (ev1) cudaEventRecord(ev1, st);
  HaloArgs h;
  h.item_base = pl.itembase.as<int>();
  h.nit = pl.nit.as<int>();
  h.scratch = scratch.as<float2>();
  h.grid = grid;
  h.nx = nx;
  h.ny = ny;
  h.npol = v.npol;
  h.nchan_img = nchan_img;
  h.tile = pl.tile;
  h.ntx = pl.ntx;
  h.nty = pl.nty;
  h.ntiles = (long long)pl.ntx * pl.nty;
  h.smax = pl.smax;
  h.P = P;
  h.slot_pol = gtile ? (long long)Pg * Pg + gtile_nthr : (long long)P * P;
  h.row = gtile ? Pg : P;
  const long long nblocks = pl.ntiles_total;
  if (nblocks > 0x7fffffffll) return YG_ERR_UNSUPPORTED;
  k_halo_sum<<<(unsigned)nblocks, 256, 0, st>>>(h);
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(cudaGetLastError());
  return YG_OK;
}

// Degrids the samples of a plan from `grid` and adds the result into vis.
int plan_degrid(Plan& pl, const VisArgs& v, float2* vis_out, const CFView& cf, const float2* grid, int nx, int ny,
                int nchan_img, const int* chan_map, DevBuf& tmp_vals, float2* carry, DevError* err,
                cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, const LearnedCF* lcf, int variant, bool alone) {
  const long long n = pl.nsamples;
  if (n == 0) return YG_OK;
  if (pl.grid_only) return YG_ERR_STATE;     // no CF-major records
  YG_CUDA_TRY(tmp_vals.ensure((size_t)n * v.npol * sizeof(float2)));
  bool done = false;
  const bool learned = lcf && lcf->w16;
  if (learned && (cf.wpad <= 0 || cf.wpad > 64 || !(v.npol == 1 || v.npol == 2 || v.npol == 4)))
    return YG_ERR_UNSUPPORTED;
  if (pl.nitems > 0 && cf.pad && cf.wpad > 0 && cf.wpad <= 128 && (v.npol == 1 || v.npol == 2 || v.npol == 4)) {
    DegridTArgs d;
    d.items = pl.items.as<int4>();
    d.rec = pl.rec.as<int4>();
    d.v = v;
    d.cf = cf;
    d.grid = grid;
    d.nx = nx;
    d.ny = ny;
    d.nchan_img = nchan_img;
    d.tile = pl.tile;
    d.ntx = pl.ntx;
    d.ntiles = (long long)pl.ntx * pl.nty;
    d.smax = pl.smax;
    d.Pg = grid_tile_stride(pl.tile, cf.wpad, pl.smax, cf.varsup != 0);
    d.Wp = cf.wpad;
    d.cfbuf = grid_cf_buffer_bytes(cf.wpad);
    d.out = tmp_vals.as<float2>();
    d.err = err;
    d.lcf = learned ? *lcf : LearnedCF{};
    d.ext = learned ? lcf->ext : nullptr;
    const int xv = d.ext ? 2 : 0;
    size_t smem;
    if (learned) {
      // records-only stages (plus the continuous inputs); the network and one
      // evaluated plane after them
      d.cfbuf = 0;
      const size_t tile = degrid_t_tile_bytes(v.npol, d.Pg), extra = learned_smem_bytes(d.Wp);
      const size_t stage = (size_t)seg_stage_bytes(0, xv) + 16;
      d.nstages = tile + extra + 2 * stage <= 227 * 1024 ? (int)std::min<size_t>(8, (227 * 1024 - tile - extra) / stage)
                                                          : 0;
      if (d.nstages == 0) return YG_ERR_UNSUPPORTED;
      smem = tile + (size_t)d.nstages * stage + extra;
    } else {
      d.nstages = degrid_t_stages(v.npol, d.Pg, d.cfbuf);
      smem = degrid_t_smem_bytes(v.npol, d.Pg, d.cfbuf, d.nstages);
    }
    d.stage_bytes = seg_stage_bytes(d.cfbuf, xv);
    // Owned segments need a ring depth that is a multiple of the tap warps:
    // segment s sits in stage s mod NST and belongs to warp s mod ncw, so then
    // every stage has one owner, which waits for the stage's fills in order.
    // With another depth, stage st also holds segments of other warps, and a
    // warp could begin waiting for the stage's next fill while the previous
    // one (another warp's, its bulk copy still in flight) had not completed:
    // the parity wait takes the incomplete phase for the one before it and
    // returns at once, and the warp reads the other segment.
    const int ncw_d = kDegridThreads / 32;
    d.own = (alone && d.nstages >= ncw_d) ? 1 : 0;
    if (d.own && !learned) {   // (the learned forms' rings hold at most ncw stages)
      d.nstages = d.nstages / ncw_d * ncw_d;
      smem = degrid_t_smem_bytes(v.npol, d.Pg, d.cfbuf, d.nstages);
    }
    if (d.nstages > 0) {
      if (ev0) cudaEventRecord(ev0, st);
      const int threads = kDegridThreads + 32;   // tap warps + the producer warp
      auto launch = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<pl.nitems, threads, smem, st>>>(d);
      };
      // 16-wide CF planes: the register-CF kernel unless variant bit 256
      // asks for k_degrid_t (both need a stage per tap warp)
      const bool regcf = !learned && d.Wp == 16 && d.nstages >= kDegridThreads / 32 && !(variant & 256);
      // bit 512: one sample per half-warp pass instead of two
      const bool sph1 = (variant & 512) != 0;
      switch (v.npol * 10 + (learned ? (d.ext ? 3 : 2) : 0)) {
        case 10: regcf ? (sph1 ? launch(k_degrid_r<1, 1>) : launch(k_degrid_r<1, 2>)) : launch(k_degrid_t<1, 0>); break;
        case 20: regcf ? (sph1 ? launch(k_degrid_r<2, 1>) : launch(k_degrid_r<2, 2>)) : launch(k_degrid_t<2, 0>); break;
        case 40: regcf ? (sph1 ? launch(k_degrid_r<4, 1>) : launch(k_degrid_r<4, 2>)) : launch(k_degrid_t<4, 0>); break;
        case 12: launch(k_degrid_t<1, 2>); break;
        case 22: launch(k_degrid_t<2, 2>); break;
        case 42: launch(k_degrid_t<4, 2>); break;
        case 13: launch(k_degrid_t<1, 3>); break;
        case 23: launch(k_degrid_t<2, 3>); break;
        default: launch(k_degrid_t<4, 3>); break;
      }
      YG_COUNT_LAUNCH();
      if (ev1) cudaEventRecord(ev1, st);
      YG_CUDA_TRY(cudaGetLastError());
      done = true;
    }
  }
  if (pl.nitems > 0 && !done) {
    DegridKArgs d;
    d.items = pl.items.as<int4>();
    d.rec = pl.rec.as<int4>();
    d.val = pl.val.as<unsigned int>();
    d.pos = pl.pos.as<unsigned int>();
    d.cfi = pl.cfi.as<int>();
    d.v = v;
    d.cf = cf;
    d.grid = grid;
    d.nx = nx;
    d.ny = ny;
    d.nchan_img = nchan_img;
    d.chan_map = chan_map;
    d.tile = pl.tile;
    d.ntx = pl.ntx;
    d.ntiles = (long long)pl.ntx * pl.nty;
    d.smax = pl.smax;
    d.P = pl.pad;
    d.out = tmp_vals.as<float2>();
    const int W = 2 * pl.smax + 1;
    const size_t tab_bytes = (size_t)W * W * sizeof(int);
    size_t smem = (size_t)v.npol * pl.pad * pl.pad * sizeof(float2) + tab_bytes;
    d.smem_grid = smem <= 200 * 1024 ? 1 : 0;
    if (!d.smem_grid) smem = tab_bytes;
    if (smem > 227 * 1024) return YG_ERR_UNSUPPORTED;
    cudaError_t e = cudaSuccess;
    if (ev0) cudaEventRecord(ev0, st);
    switch (v.npol) {
      case 1: {
        auto k = k_degrid<1>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<pl.nitems, kDegridThreads, smem, st>>>(d);
        YG_COUNT_LAUNCH();
        break;
      }
      case 2: {
        auto k = k_degrid<2>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<pl.nitems, kDegridThreads, smem, st>>>(d);
        YG_COUNT_LAUNCH();
        break;
      }
      case 4: {
        auto k = k_degrid<4>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<pl.nitems, kDegridThreads, smem, st>>>(d);
        YG_COUNT_LAUNCH();
        break;
      }
      default:
        return YG_ERR_UNSUPPORTED;
    }
    if (ev1) cudaEventRecord(ev1, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return YG_ERR_CUDA;
  }
  // write-back with the reference's carried value for off-grid samples; the
  // loop-order predecessor scan depends only on the plan, so it is computed
  // on the first degridding pass of a plan and kept
  YG_CUDA_TRY(pl.order_prev.ensure((size_t)n * 4 * 2));
  int* marks = pl.order_prev.as<int>();
  int* prev = marks + n;
  if (!pl.prev_ready) {
    k_order_marks<<<grid_dim(n, 256), 256, 0, st>>>(pl.status.as<unsigned char>(), pl.nrow, pl.nchan, 3, marks);
    YG_COUNT_LAUNCH();
    YG_CUDA_TRY(pl.sort_tmp.ensure(std::max(scan_tmp_bytes(n), pl.sort_tmp.bytes)));
    YG_CUDA_TRY(scan_i32(marks, prev, n, SCAN_MAX, false, pl.sort_tmp.p, pl.sort_tmp.bytes, st));
    pl.prev_ready = true;
  }
  k_degrid_writeback<<<grid_dim(n, 256), 256, 0, st>>>(pl.status.as<unsigned char>(), prev, tmp_vals.as<float2>(),
                                                       carry, pl.nrow, pl.nchan, v.npol, vis_out);
  YG_COUNT_LAUNCH();
  k_update_carry<<<1, 32, 0, st>>>(prev + (n - 1), pl.nrow, pl.nchan, v.npol, tmp_vals.as<float2>(), 0, carry);
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(cudaGetLastError());
  return YG_OK;
}

// Continuous learned CF, once per plan: for every sorted sample the residue of
// its fractional offsets beyond the tabulated fraction, ru = (t - nint(t)) / os
// with t = os (iu - u f / (c cellu)) and likewise rv, and its own w (minus its
// w-stack's w term) over wnorm.  Neither residue changes the indices: they
// only feed the network.
__global__ void k_learned_inputs(const int4* __restrict__ rec, const unsigned long long* __restrict__ key,
                                 long long nvalid, const double* __restrict__ uvw, const double* __restrict__ freq,
                                 long long nrow, double cellu, double cellv, int os, int mbits, int ncf,
                                 long long ntiles, int nchan_img, const double* __restrict__ wstack, double wnorm,
                                 float4* __restrict__ out) {
  const double C = 299792458.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid; i += (long long)gridDim.x * blockDim.x) {
    const long long s = rec[i].w;
    const long long row = s % nrow;
    const int chan = (int)(s / nrow);
    const double f = freq[chan];
    const double us = uvw[3 * row] * f / (C * cellu);
    const double vs = uvw[3 * row + 1] * f / (C * cellv);
    const double tu = os * ((double)nint_d(us) - us);
    const double tv = os * ((double)nint_d(vs) - vs);
    double w = uvw[3 * row + 2] * f / C;
    if (wstack) {
      const long long gc = (long long)((key[i] >> mbits) / (unsigned long long)ncf) / ntiles;
      w -= wstack[gc / nchan_img];
    }
    out[i] = make_float4((float)((tu - (double)nint_d(tu)) / os), (float)((tv - (double)nint_d(tv)) / os),
                         (float)(w / wnorm), 0.f);
  }
}

int plan_learned_inputs(Plan& pl, const double* uvw, const double* freq, double cellu, double cellv, int os,
                        int nchan_img, const double* wstack, double wnorm, cudaStream_t st) {
  if (pl.ext_ready) return YG_OK;
  YG_CUDA_TRY(pl.ext.ensure_headroom((size_t)std::max(1ll, pl.nvalid) * sizeof(float4)));
  if (pl.nvalid > 0) {
    k_learned_inputs<<<grid_dim(pl.nvalid, 256), 256, 0, st>>>(
        pl.rec.as<int4>(), pl.key.as<unsigned long long>(), pl.nvalid, uvw, freq, pl.nrow, cellu, cellv, os, pl.mbits,
        pl.ncf, (long long)pl.ntx * pl.nty, nchan_img, wstack, wnorm, pl.ext.as<float4>());
    YG_COUNT_LAUNCH();
    YG_CUDA_TRY(cudaGetLastError());
  }
  pl.ext_ready = true;
  return YG_OK;
}

// grid mode: itsImagePolFrameVis ends as the last used (flag-free, mapped)
// sample's visibility in loop order.
int plan_grid_carry(Plan& pl, const VisArgs& v, float2* carry, cudaStream_t st) {
  const long long n = pl.nsamples;
  if (n == 0 || v.psf || v.pcf) return YG_OK;
  YG_CUDA_TRY(pl.last.ensure(sizeof(int)));
  YG_CUDA_TRY(cudaMemsetAsync(pl.last.p, 0xff, sizeof(int), st));
  k_last_marked<<<grid_dim(n, 256), 256, 0, st>>>(pl.status.as<unsigned char>(), pl.nrow, pl.nchan, 1,
                                                  pl.last.as<int>());
  YG_COUNT_LAUNCH();
  k_update_carry<<<1, 32, 0, st>>>(pl.last.as<int>(), pl.nrow, pl.nchan, v.npol, v.vis, 1, carry);
  YG_COUNT_LAUNCH();
  YG_CUDA_TRY(cudaGetLastError());
  return YG_OK;
}

}  // namespace yg
