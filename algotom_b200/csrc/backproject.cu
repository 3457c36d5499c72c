// Linear-interpolation back-projection (pixel-driven gather), sm_100a.
//
// Same mathematics as algotom's back-projectors
// (algotom/rec/reconstruction.py:156-190, 229-264, 307-359): pixel (y, x)
// of an ncol x ncol slice reads detector position
//     p = (x - ic) cos(-a) + (y - ic) sin(-a) + center,  ic = (ncol - 1) / 2
// and adds s[d] + (s[d+1] - s[d]) (p - d), d = floor(p), when
// 0 <= p <= ncol - 1; outside it adds nothing, or with edge padding the
// nearest edge sample.
//
// Work decomposition.  A CTA of 256 threads owns a pixel tile of S slices
// that share angles and centre, and walks the angles in chunks.  For every
// angle of a chunk the tile only sees a window of kWin detector bins (its
// footprint is at most (TX-1)|cos| + (TY-1)|sin| + 2 bins wide), so the CTA
// stages just that window, per slice, into shared memory as interpolation
// pairs
//     (a_j, D_j) = (s[lo+j] - (j-H) D_j, s[lo+j+1] - s[lo+j]),  H = kWin/2
// so that the value at the window-centred local position q = p - lo - H,
// bin j = floor(q) + H, is the single FMA a_j + D_j q.  With S >= 2 the pairs
// of two slices sit in one 16-byte word (a_0, a_1, D_0, D_1), one plane per
// slice pair so that neighbouring bins are 16 bytes apart (conflict-free
// quarter-warp LDS.128): one LDS.128, one packed fma.rn.f32x2 and one packed
// add.rn.f32x2 update two slices, and the position, floor and address work
// is shared by all S slices.
//
// Staging is pipelined: while chunk k accumulates from one of two pairs
// buffers, chunk k + 1's raw detector windows stream into shared memory;
// then k + 1's pairs are built into the other buffer, and after one CTA
// barrier k + 2's windows are requested into the single raw buffer.  For CTAs
// of 2 or 4 slices whose rows are 16-byte aligned, each angle's window of
// all S slices is one TMA box load (cp.async.bulk.tensor.3d over the
// [angle][slice][bin] array, zero fill outside it) issued by one thread per
// angle, completing on an mbarrier per buffer.  Single-slice CTAs (and the
// persistent batch kernel) use 16-byte cp.async; other layouts 4-byte
// cp.async, or plain loads for 16-bit storage.  A short pass then turns the
// windows into pairs.
//
// Bounds: bins outside the detector hold (0, 0) (or the edge value with
// D = 0 under edge padding), which reproduces the reference wherever the
// interpolant is continuous.  The two detector edges of FBP (no edge
// padding) are discontinuities: angles whose tile footprint reaches either
// edge take a checked path (a CTA-uniform branch) that tests every position
// against both edges and re-decides, in FP64 with the reference's own
// expression, any position within 2e-3 bins of an edge -- at exactly 90
// degrees whole pixel rows sit 1e-8 bins from position 0, which no FP32 local
// coordinate can resolve.
//
// Positions: the tile-origin position is formed in FP64 per (tile, angle)
// from FP64 trigonometry of the float32-rounded angle; each thread adds its
// in-tile offset in FP32, so q is accurate to ~1e-5 bins at any image size.
// floor(q) is one round-down add of 1.5 * 2^23, whose bit pattern is the
// shared-memory index.
//
// Accumulation: FP32 partial sums over each chunk of angles, added across
// chunks with Kahan compensation (the single-slice kernel can instead
// compensate every angle).  One warp instruction covers an 8 x 4 pixel
// block, whose 32 lanes read a run of about 9 neighbouring bins.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched at run time)
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <type_traits>

#include "common.cuh"

namespace {

// polls of a staging mbarrier (64 ns apart) before a CTA gives up on a
// window load: about 70 ms, against microseconds in normal operation
constexpr int kWaitPolls = 1 << 20;
// set (bit 0) by a CTA whose staging wait ran out; read by atb_backproject_status
__device__ int g_bp_status;

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr float kEdgeTol = 2e-3f;  // bins; FP32 error of q is < 3e-5

// Tile geometry per slices-per-CTA S and variant V.  Warp tile = (8 PX) x
// (4 PY) pixels, CTA = WX x WY warps; kWin >= (TX-1)+(TY-1)/sqrt(2)... i.e.
// the tile's largest footprint sqrt((TX-1)^2 + (TY-1)^2) plus 4 bins.
// Variant 1 of the single-slice geometry is a 32 x 32 tile on 128 threads:
// less shared memory and fewer registers, so more CTAs share an SM (small
// images, uneven batches); the autotuner chooses between the variants.
template <int S, int V = 0> struct Geo;
template <> struct Geo<1, 0> {
  static constexpr int PX = 4, PY = 4, WX = 2, WY = 4, kChunk = 32, kWin = 96, kThreads = 256, kMinBlocks = 2;
};
template <> struct Geo<1, 1> {
  static constexpr int PX = 2, PY = 4, WX = 2, WY = 2, kChunk = 32, kWin = 48, kThreads = 128, kMinBlocks = 4;
};
template <> struct Geo<2, 0> {
  static constexpr int PX = 2, PY = 4, WX = 4, WY = 2, kChunk = 16, kWin = 80, kThreads = 256, kMinBlocks = 2;
};
template <> struct Geo<4, 0> {
  static constexpr int PX = 2, PY = 4, WX = 4, WY = 2, kChunk = 16, kWin = 80, kThreads = 256, kMinBlocks = 2;
};

struct BPArgs {
  const void *sino;
  long long srs, sss;
  int nrow, nslice, ncol;
  int slice_base;  // first slice of this launch
  const double2 *trig;
  double center;
  int edge_pad;
  double mask_r2;
  float scale;
  float *out;
  long long ors, oss;
  int vec16;  // rows 16-byte aligned: stage by TMA (tma) or 16-byte cp.async
  int tma;    // the kernel's tensor map describes sino: stage windows by TMA
  int spacing;  // centre-group launches: slice m is centre center + m spacing
                // of the one sinogram (sss = 0)
  int slope;  // back-project the interpolant's slope D_j instead of its value
  int wait_polls;  // polls before a staging wait gives up (kWaitPolls)
  int inject;      // test only: CTA (0, 0, 0) arms its first staging wait
                   // for 16 bytes more than its copies deliver
};

struct __align__(16) AngleParam {
  float qbase;  // local position of the tile-origin pixel, q = p - lo - H
  float c, s;   // cos(-a), sin(-a) in FP32 for in-tile offsets
  float qmax;   // local position of detector bin ncol - 1
  float qlo;    // local position of detector bin 0
  int j0;       // window index of detector bin 0
  double c64, s64;  // FP64 trigonometry, for the exact edge decision
};

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

// packed FP32 pairs (Blackwell f32x2 arithmetic)
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
// acc += d * q + a in both lanes
__device__ __forceinline__ void fma_acc2(unsigned long long &acc, unsigned long long av, unsigned long long dv,
                                         unsigned long long q) {
  unsigned long long v;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(v) : "l"(dv), "l"(q), "l"(av));
  asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc) : "l"(v));
}

// Tensor memory (TMEM, 128 lanes x 512 columns of 32-bit cells per SM)
// holds the compensated running totals between chunk folds, which keeps
// them out of the registers of the accumulation loop.  Warp w of a CTA
// reaches lanes 32 (w % 4) .. 32 (w % 4) + 31 only; every thread uses the
// cells of its own lane.  An address is (lane << 16) | column.  Each
// transfer waits for its own completion, so the registers are free after it.
template <int N> __device__ __forceinline__ void tmem_ld(uint32_t taddr, float *r);
template <int N> __device__ __forceinline__ void tmem_st(uint32_t taddr, const float *r);
template <> __device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7]), "=f"(r[8]), "=f"(r[9]), "=f"(r[10]), "=f"(r[11]), "=f"(r[12]), "=f"(r[13]), "=f"(r[14]), "=f"(r[15])
      : "r"(taddr)
      : "memory");
}
template <> __device__ __forceinline__ void tmem_st<16>(uint32_t taddr, const float *r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};\n\t"
      "tcgen05.wait::st.sync.aligned;"
      :
      : "r"(taddr), "f"(r[0]), "f"(r[1]), "f"(r[2]), "f"(r[3]), "f"(r[4]), "f"(r[5]), "f"(r[6]), "f"(r[7]), "f"(r[8]), "f"(r[9]), "f"(r[10]), "f"(r[11]), "f"(r[12]), "f"(r[13]), "f"(r[14]), "f"(r[15])
      : "memory");
}
template <> __device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7]), "=f"(r[8]), "=f"(r[9]), "=f"(r[10]), "=f"(r[11]), "=f"(r[12]), "=f"(r[13]), "=f"(r[14]), "=f"(r[15]), "=f"(r[16]), "=f"(r[17]), "=f"(r[18]), "=f"(r[19]), "=f"(r[20]), "=f"(r[21]), "=f"(r[22]), "=f"(r[23]), "=f"(r[24]), "=f"(r[25]), "=f"(r[26]), "=f"(r[27]), "=f"(r[28]), "=f"(r[29]), "=f"(r[30]), "=f"(r[31])
      : "r"(taddr)
      : "memory");
}
template <> __device__ __forceinline__ void tmem_st<32>(uint32_t taddr, const float *r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};\n\t"
      "tcgen05.wait::st.sync.aligned;"
      :
      : "r"(taddr), "f"(r[0]), "f"(r[1]), "f"(r[2]), "f"(r[3]), "f"(r[4]), "f"(r[5]), "f"(r[6]), "f"(r[7]), "f"(r[8]), "f"(r[9]), "f"(r[10]), "f"(r[11]), "f"(r[12]), "f"(r[13]), "f"(r[14]), "f"(r[15]), "f"(r[16]), "f"(r[17]), "f"(r[18]), "f"(r[19]), "f"(r[20]), "f"(r[21]), "f"(r[22]), "f"(r[23]), "f"(r[24]), "f"(r[25]), "f"(r[26]), "f"(r[27]), "f"(r[28]), "f"(r[29]), "f"(r[30]), "f"(r[31])
      : "memory");
}

// Columns of TMEM a CTA of BPCfg<T, S, V> takes: two cells (total,
// compensation) per pixel and slice for each thread, times the warps that
// share a lane quarter, rounded up to a power of two >= 32.
constexpr int tmem_cols(int cells_per_thread, int threads) {
  int need = cells_per_thread * (threads / 128), c = 32;
  while (c < need) c *= 2;
  return c;
}

// Warp 0 allocates kCols columns for the CTA (and gives up the right to
// allocate more, so other CTAs of the SM never wait on this one); every
// thread returns the base address.  All threads of the CTA must call it.
template <int kCols>
__device__ __forceinline__ uint32_t tmem_alloc_cta(uint32_t *slot) {
  if (threadIdx.x < 32) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(slot);
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n\t"
        "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::"r"(a),
        "n"(kCols)
        : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *reinterpret_cast<volatile uint32_t *>(slot);
}

// Warp 0 frees the CTA's columns once every thread is done with them.  All
// threads of the CTA must call it.
template <int kCols>
__device__ __forceinline__ void tmem_free_cta(uint32_t base) {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (threadIdx.x < 32) {
    asm volatile(
        "tcgen05.fence::after_thread_sync;\n\t"
        "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base),
        "n"(kCols)
        : "memory");
  }
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
// mbarrier and TMA helpers for the window staging
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// waits for the phase of the given parity to complete; false if it has not
// after kWaitPolls polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int polls) {
  const uint32_t addr = smem_u32(bar);
  for (int n = 0; n < polls; ++n) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(64);
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// box (x, y, z) of the tensor map into shared memory, completing on bar
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T, int S, int V = 0>
struct BPCfg {
  using G = Geo<S, V>;
  static constexpr int kThreads = G::kThreads, kMinBlocks = G::kMinBlocks;
  static constexpr int PX = G::PX, PY = G::PY, WX = G::WX;
  static constexpr int TX = 8 * PX * G::WX, TY = 4 * PY * G::WY;
  static constexpr int kChunk = G::kChunk, kWin = G::kWin, kHalf = kWin / 2;
  // raw window: elements of T from a start rounded down to a 16-byte vector
  static constexpr int kVecElems = 16 / (int)sizeof(T);
  static constexpr int kRaw = ((kWin + 1 + (kVecElems - 1) + (kVecElems - 1)) / kVecElems) * kVecElems;
  // bfloat16 storage with S >= 2 keeps 16-bit (value, difference) pairs in
  // shared memory: 4 bytes per bin and slice instead of 8 (bfloat16 widens
  // to FP32 with one shift; float16 would need conversions, which cost more
  // issue slots than the halved shared-memory traffic saves, so float16
  // stages FP32 pairs)
  static constexpr bool kHalfPairs = std::is_same<T, __nv_bfloat16>::value && S >= 2;
  static constexpr int kPairBytes = (kHalfPairs ? 4 : 8) * S;  // per bin: S pairs
  static constexpr size_t kPairsSmem = (size_t)kChunk * kWin * kPairBytes;
  // one angle's S windows: a TMA box of S x kRaw elements, in a slot padded
  // to a multiple of 128 bytes (TMA destinations are 128-byte aligned)
  static constexpr int kBoxBytes = S * kRaw * (int)sizeof(T);
  static constexpr int kRawSlot = ((kBoxBytes + 127) / 128) * 128 / (int)sizeof(T);
  // pairs double-buffered (one chunk accumulates while the next is built),
  // raw windows single-buffered (consumed before the next chunk's arrive)
  static constexpr size_t kRawSmem = (size_t)kChunk * kRawSlot * sizeof(T);
  static constexpr size_t kSmem = 2 * kPairsSmem + kRawSmem + 128;  // + slack to align the raw region
  // compensated totals in TMEM: kAcc accumulators per thread, as (total,
  // compensation) cells in 2 kAcc columns; moved kXfer accumulators at a time
  static constexpr int kAcc = PX * G::PY * S;
  static constexpr int kXfer = kAcc % 16 == 0 ? 16 : 8;
  static constexpr int kTmemCols = tmem_cols(2 * kAcc, kThreads);
  static_assert(kThreads % 128 == 0 && kAcc % 8 == 0, "TMEM layout");
};

// One CTA's work: the TX x TY pixel tile (bx, by) of the slice group bz.
// Every thread of the CTA must call it (it synchronises).  tmem is the
// base of the CTA's K::kTmemCols TMEM columns (chunked Kahan only).
// kGroup: the launch's slices are candidate centres center + m spacing of
// ONE sinogram (a centre search).  Slice m at centre c + m spacing sees the
// same local positions q as the CTA's first slice on a source row shifted
// by m spacing bins, so a CTA stages one row segment covering all its
// slices and builds each slice's pairs from it at that shift; the
// accumulation is the stacked one.  Edge angles decide the detector range
// per slice.
__host__ __device__ constexpr int group_segment(int win, int s, int spacing, int vec) {
  return ((win + (s - 1) * spacing + 3 * vec - 1) / vec) * vec;
}

template <typename T, int S, bool kPerAngleKahan, int V = 0, bool kGroup = false>
__device__ __forceinline__ void bp_tile(const BPArgs &a, int bx, int by, int bz, unsigned char *smem,
                                        uint32_t tmem, const CUtensorMap *tmap) {
  using K = BPCfg<T, S, V>;
  constexpr int kThreads = K::kThreads;
  constexpr int PX = K::PX, PY = K::PY, TX = K::TX, TY = K::TY;
  constexpr int kChunk = K::kChunk, kWin = K::kWin, kHalf = K::kHalf, kRaw = K::kRaw;
  constexpr int NP = (S + 1) / 2;  // packed accumulator words per pixel

  // two buffers of pairs, S == 1: [kChunk][kWin] float2; else
  // [kChunk][S/2][kWin] float4; chunk k uses buffer k & 1
  unsigned char *pairs_buf = smem;
  // [kChunk] slots of [S][kRaw] (one centre group row: [seglen]), on a
  // 128-byte boundary
  const unsigned raw_off = 2 * (unsigned)K::kPairsSmem;
  T *raw = reinterpret_cast<T *>(smem + raw_off + ((128u - (smem_u32(smem + raw_off) & 127u)) & 127u));
  __shared__ __align__(8) uint64_t raw_bar;  // TMA completion of the raw windows (phase k & 1: chunk k)
  // per-angle parameters in three slots (chunk k: slot k % 3), so chunk
  // k + 2's are written while chunk k accumulates and k + 1's are in use
  __shared__ AngleParam prm[3][kChunk];
  __shared__ int lo_s[3][kChunk];
  __shared__ int flag_s[3][kChunk];  // bit 0: skip angle, bit 1: checked path

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int x0 = bx * TX, y0 = by * TY;
  const int slice0 = a.slice_base + bz * S;
  const int nsl = min(S, a.nslice - slice0);  // live slices of this CTA
  const bool use_tma = a.tma != 0;
  const int ncol = a.ncol;
  const T *sino = reinterpret_cast<const T *>(a.sino) + slice0 * a.sss;
  // centre-group launches: this CTA's first centre, the shift between its
  // slices and the length of the row segment it stages
  const int gsp = kGroup ? a.spacing : 0;
  const double ctr = kGroup ? a.center + (double)slice0 * (double)gsp : a.center;
  const int seglen = kGroup ? group_segment(kWin, S, gsp, K::kVecElems) : kRaw;

  // thread -> pixel offsets inside the tile: warp (wx, wy) covers
  // (8 PX) x (4 PY) pixels, lane (lx, ly) an 8 x 4 block replicated PX x PY
  const int tx = (warp % K::WX) * (8 * PX) + (lane & 7);
  const int ty = (warp / K::WX) * (4 * PY) + (lane >> 3);

  // accumulators: FP32 chunk partials (packed two slices per word when
  // S >= 2) and the compensated running totals, in registers for per-angle
  // Kahan and in TMEM (accumulator n = (b PX + c) S + k at columns 2n,
  // 2n + 1 of this thread's span) for chunked Kahan
  float accf[PY][PX];
  unsigned long long acc2[PY][PX][NP];
  float sum[PY][PX][S], comp[PY][PX][S];
#pragma unroll
  for (int b = 0; b < PY; ++b)
#pragma unroll
    for (int c = 0; c < PX; ++c) {
      accf[b][c] = 0.f;
#pragma unroll
      for (int g = 0; g < NP; ++g) acc2[b][c][g] = 0ull;
#pragma unroll
      for (int k = 0; k < S; ++k) { sum[b][c][k] = 0.f; comp[b][c][k] = 0.f; }
    }
  constexpr int kAcc = K::kAcc, kXfer = K::kXfer;
  const uint32_t tm = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * 2 * kAcc);
  // chunk partial of accumulator n
  auto partial = [&](int n) -> float {
    const int k = n % S, c = (n / S) % PX, b = n / (S * PX);
    if constexpr (S == 1) {
      return accf[b][c];
    } else {
      float lo, hi;
      unpack2(acc2[b][c][k / 2], lo, hi);
      return (k & 1) ? hi : lo;
    }
  };
  if constexpr (!kPerAngleKahan) {
    float z[2 * kXfer];
#pragma unroll
    for (int i = 0; i < 2 * kXfer; ++i) z[i] = 0.f;
#pragma unroll
    for (int n0 = 0; n0 < kAcc; n0 += kXfer) tmem_st<2 * kXfer>(tm + 2 * n0, z);
  }

  const double ic = 0.5 * (double)(ncol - 1);
  const int nchunk = (a.nrow + kChunk - 1) / kChunk;

  // per-angle window and local-position parameters of chunk k, FP64
  auto params = [&](int k, int buf) {
    if (tid < kChunk) {
      const int i = k * kChunk + tid;
      int flag = 1, lo = 0;
      AngleParam p = {0.f, 0.f, 0.f, 0.f, 0.f, 0, 0.0, 0.0};
      if (i < a.nrow) {
        const double2 cs = a.trig[i];
        const double P0 = ((double)x0 - ic) * cs.x + ((double)y0 - ic) * cs.y + ctr;
        const double ec = (double)(TX - 1) * cs.x, es = (double)(TY - 1) * cs.y;
        // non-finite trig (rejected by the host) is skipped, never indexed
        if (isfinite(P0) && isfinite(ec) && isfinite(es)) {
          const double pmin = P0 + fmin(0.0, ec) + fmin(0.0, es);
          const double pmax = P0 + fmax(0.0, ec) + fmax(0.0, es);
          // highest position of any slice (a centre group's last slice sits
          // (S - 1) spacing bins further)
          const double pmax_all = pmax + (double)((S - 1) * gsp);
          lo = (int)floor(pmin) - 1;
          p.qbase = (float)(P0 - (double)(lo + kHalf));
          p.c = (float)cs.x;
          p.s = (float)cs.y;
          p.qmax = (float)((double)(ncol - 1) - (double)(lo + kHalf));
          p.qlo = (float)(-(lo + kHalf));
          p.j0 = -lo;
          p.c64 = cs.x;
          p.s64 = cs.y;
          flag = 0;
          if (a.slope) {
            // slope mode is continuous (edges smoothed over one bin)
            if (pmin > (double)ncol + 1e-2 || pmax < -1.0 - 1e-2) flag = 1;
          } else if (!a.edge_pad) {
            if (pmin > (double)(ncol - 1) + 1e-2 || pmax_all < -1e-2) flag = 1;
            else if (pmin < 1e-2 || pmax_all > (double)(ncol - 1) - 1e-2) flag = 2;
          }
        }
      }
      prm[buf][tid] = p;
      lo_s[buf][tid] = lo;
      flag_s[buf][tid] = flag;
    }
  };

  // Staging work is split by angle: kTPA threads per angle of the chunk,
  // each taking every kTPA-th bin of that angle's window.
  constexpr int kTPA = kThreads / kChunk;
  constexpr int kJPT = kWin / kTPA;
  static_assert(kThreads % kChunk == 0 && kWin % kTPA == 0, "staging split");
  const int s_ai = tid / kTPA, s_jl = tid % kTPA;
  const int ncol1 = ncol - 1;
  const long long srs = a.srs, sss = a.sss;
  const bool edge_pad = a.edge_pad, slope = a.slope, vec16 = a.vec16;
  if (use_tma && tid == 0) {  // one arrival per angle of a chunk
    mbar_init(&raw_bar, kChunk);
    mbar_init_fence();
  }

  // raw windows (and, for edge padding or slope mode, the two edge samples)
  // of chunk k into raw[buf], from a start rounded down to a 16-byte vector.
  // Aligned rows stream in with 16-byte cp.async; float32 rows that are not
  // 16-byte aligned use 4-byte cp.async, 16-bit ones plain loads.  Elements
  // outside the detector row are never read.
  auto issue_raw = [&](int k, int buf) {
    constexpr int kV = K::kVecElems;
    if (use_tma && tid < kChunk) {  // thread t: the box of angle t, or a bare arrival
      const int it = k * kChunk + tid;
      if (it < a.nrow && !(flag_s[buf][tid] & 1)) {
        const int lo = lo_s[buf][tid];
        const int base = (lo / kV - (lo % kV < 0)) * kV;  // a 16-byte multiple, as TMA requires
        fence_proxy_async_smem();
        unsigned bytes = (unsigned)(kGroup ? seglen * (int)sizeof(T) : K::kBoxBytes);
        if (a.inject && k == 0 && tid == 0 && bx == 0 && by == 0 && bz == 0) bytes += 16u;
        mbar_arrive_expect_tx(&raw_bar, bytes);
        tma_load_3d(raw + (size_t)tid * K::kRawSlot, tmap, base, kGroup ? 0 : slice0, it, &raw_bar);
      } else {
        mbar_arrive(&raw_bar);
      }
    }
    const int i = k * kChunk + s_ai;
    if (i < a.nrow && !(flag_s[buf][s_ai] & 1)) {
      const int base = (lo_s[buf][s_ai] / kV - (lo_s[buf][s_ai] % kV < 0)) * kV;  // floor to a vector
      const T *src = sino + i * srs;
      T *rb = raw + (size_t)s_ai * K::kRawSlot;
      if (use_tma) {
        // the window arrives by TMA
      } else if (vec16) {
        // rows of S slices, or a centre group's one row segment
        const int kVec = seglen / kV, nrows = kGroup ? 1 : nsl;
        for (int idx = s_jl; idx < (kGroup ? 1 : S) * kVec; idx += kTPA) {
          const int ks = idx / kVec, v = idx - ks * kVec;
          const int d = base + kV * v;
          if (ks < nrows && d >= 0 && d < ncol)  // ncol % kV == 0: a vector is in or out
            cp_async16(rb + ks * kRaw + kV * v, src + ks * sss + d);
        }
      } else if constexpr (sizeof(T) == 4) {
        const int nrows = kGroup ? 1 : nsl;
        for (int idx = s_jl; idx < (kGroup ? 1 : S) * seglen; idx += kTPA) {
          const int ks = idx / seglen, v = idx - ks * seglen;
          const int d = base + v;
          if (ks < nrows && d >= 0 && d < ncol) cp_async4(rb + ks * kRaw + v, src + ks * sss + d);
        }
      } else {
        const int nrows = kGroup ? 1 : nsl;
        for (int idx = s_jl; idx < (kGroup ? 1 : S) * seglen; idx += kTPA) {
          const int ks = idx / seglen, v = idx - ks * seglen;
          const int d = base + v;
          if (ks < nrows && d >= 0 && d < ncol) rb[ks * kRaw + v] = src[ks * sss + d];
        }
      }
    }
    cp_async_commit();
  };

  // chunk k's windows -> interpolation pairs (skipped angles are left as
  // they are: the accumulation never reads them)
  auto make_pairs = [&](int k, int buf, int pb) {
    unsigned char *pairs = pairs_buf + (size_t)pb * K::kPairsSmem;
    const int i = k * kChunk + s_ai;
    if (i >= a.nrow || (flag_s[buf][s_ai] & 1)) return;
    const int lo = lo_s[buf][s_ai];
    constexpr int kV = K::kVecElems;
    const int base = (lo / kV - (lo % kV < 0)) * kV;
    // every d and d+1 of the window inside [0, ncol-1] with d <= ncol-2
    // (slope mode: also clear of the smoothed edges at bins 0 and ncol-2)
    const int span = (S - 1) * gsp;  // a centre group's last slice reads span bins further
    const bool interior =
        slope ? (lo >= 1 && lo + kWin <= ncol1 - 1) : (lo >= 0 && lo + kWin + span <= ncol1);
    const T *rb = raw + (size_t)s_ai * K::kRawSlot;
    const T *src = sino + i * srs;  // this angle's rows (edge samples)
    // detector sample x (0 <= x <= ncol-1) of slice ks
    auto val = [&](int ks, int x) -> float {
      const int r = x - base;
      if (r >= 0 && r < seglen) return atb::to_float(rb[(kGroup ? 0 : ks * kRaw) + r]);
      return atb::load_as_float(src + ks * sss + (x == 0 ? 0 : ncol1));  // clamped edge sample
    };
#pragma unroll 2
    for (int t = 0; t < kJPT; ++t) {
      const int j = s_jl + kTPA * t;
      const float jc = (float)(j - kHalf);
      float av[S], dv[S];
#pragma unroll
      for (int ks = 0; ks < S; ++ks) {
        // detector bin of window index j for slice ks (shifted in a group)
        const int d = lo + j + ks * gsp;
        float v = 0.f, w = 0.f;
        if (ks < nsl) {
          if (interior) {
            const T *rk = rb + (kGroup ? 0 : ks * kRaw);
            v = atb::to_float(rk[d - base]);
            w = atb::to_float(rk[d + 1 - base]) - v;
          } else if (slope) {
            // derivative in p of the back-projected interpolant with its two
            // edge steps (+s[0] at p = 0, -s[ncol-1] at p = ncol-1) smoothed
            // over one bin: on bin d, value A + B f with f = p - d; stored
            // below as (A, B) in the (value, difference) slots
            float A = 0.f, B = 0.f;
            if (d >= 0 && d < ncol1) A = val(ks, d + 1) - val(ks, d);
            if (d == -1 || d == 0) {
              const float e0 = val(ks, 0);
              if (d == -1) B += e0;
              else { A += e0; B -= e0; }
            }
            if (d == ncol1 - 1 || d == ncol1) {
              const float e1 = val(ks, ncol1);
              if (d == ncol1 - 1) B -= e1;
              else { A -= e1; B += e1; }
            }
            v = A;
            w = B;
          } else if (edge_pad) {
            const int d0 = min(max(d, 0), ncol1), d1 = min(max(d + 1, 0), ncol1);
            v = val(ks, d0);
            w = d1 == d0 ? 0.f : val(ks, d1) - v;
          } else if (d >= 0 && d < ncol1) {
            v = val(ks, d);
            w = val(ks, d + 1) - v;
          } else if (d == ncol1) {
            v = val(ks, d);  // last bin: its value only at p = ncol-1
          }
        }
        if (slope && interior) {  // slope of the interpolant, constant per bin
          av[ks] = w;
          dv[ks] = 0.f;
        } else {  // value v + w f on bin d, f = p - d = q - (j - H)
          av[ks] = fmaf(-jc, w, v);
          dv[ks] = w;
        }
      }
      if constexpr (K::kHalfPairs) {
        // (value, difference) of two slices as two 32-bit words; the value
        // is v + D f with f = p - d, so store v itself (not the centred a)
        uint2 *p2 = reinterpret_cast<uint2 *>(pairs) + (size_t)s_ai * (S / 2) * kWin + j;
#pragma unroll
        for (int g = 0; g < S / 2; ++g) {
          float v0 = av[2 * g] + jc * dv[2 * g], v1 = av[2 * g + 1] + jc * dv[2 * g + 1];
          if (slope && interior) { v0 = av[2 * g]; v1 = av[2 * g + 1]; }
          p2[g * kWin] = make_uint2(atb::pack_pair<T>(v0, v1), atb::pack_pair<T>(dv[2 * g], dv[2 * g + 1]));
        }
      } else if constexpr (S == 1) {
        reinterpret_cast<float2 *>(pairs)[s_ai * kWin + j] = make_float2(av[0], dv[0]);
      } else {
        float4 *p4 = reinterpret_cast<float4 *>(pairs) + (size_t)s_ai * (S / 2) * kWin + j;
#pragma unroll
        for (int g = 0; g < S / 2; ++g)
          p4[g * kWin] = make_float4(av[2 * g], av[2 * g + 1], dv[2 * g], dv[2 * g + 1]);
      }
    }
  };

  // Prologue: chunk 0's windows and pairs, chunk 1's parameters and windows
  // in flight.  Then per chunk k: accumulate k from pairs buffer k & 1;
  // wait for k + 1's windows; write k + 2's parameters; build k + 1's
  // pairs into the other buffer; one barrier; request k + 2's windows.
  // (cp.async staging adds a barrier after its wait: other threads' copies.)
  params(0, 0);
  __syncthreads();
  issue_raw(0, 0);
  bool late = false;
  if (use_tma) late = !mbar_wait(&raw_bar, 0u, a.wait_polls);
  else cp_async_wait_all();
  __syncthreads();
  if (nchunk > 1) params(1, 1);
  make_pairs(0, 0, 0);
  bool stalled = __syncthreads_or(late);  // pairs(0), params(1) visible; raw free
  int pending = 0;                          // chunk whose windows are awaited
  if (!stalled && nchunk > 1) issue_raw(1, 1);

  for (int k = 0; k < nchunk && !stalled; ++k) {
    const int buf = k % 3;
    const unsigned char *pairs = pairs_buf + (size_t)(k & 1) * K::kPairsSmem;
    // accumulate chunk k
    const int nang = min(kChunk, a.nrow - k * kChunk);
    for (int ai = 0; ai < nang; ++ai) {
      const int flag = flag_s[buf][ai];
      if (flag & 1) continue;
      const AngleParam p = prm[buf][ai];
      const float qt = fmaf((float)tx, p.c, fmaf((float)ty, p.s, p.qbase));
      const float c8 = 8.f * p.c, s4 = 4.f * p.s;
      // this angle's pairs, indexed by floor(q) (window centre at 0)
      const unsigned char *w = pairs + ((size_t)ai * kWin + kHalf) * K::kPairBytes;
      if constexpr (S > 1) w = pairs + ((size_t)ai * (S / 2) * kWin + kHalf) * (K::kHalfPairs ? 8 : 16);
      auto body = [&](auto checked_tag) {
        constexpr bool kChecked = decltype(checked_tag)::value;
#pragma unroll
        for (int b = 0; b < PY; ++b) {
          const float qr = fmaf((float)b, s4, qt);
#pragma unroll
          for (int c = 0; c < PX; ++c) {
            const float q = fmaf((float)c, c8, qr);
            const float tq = __fadd_rd(q, kMagic);
            int j = __float_as_int(tq) - kMagicBits;
            bool inr = true;
            bool moved = false;
            if constexpr (kChecked && kGroup && S > 1 && !K::kHalfPairs) {
              // centre group near a detector edge: each slice has its own
              // range [0, ncol - 1] in window coordinates, shifted by its
              // spacing, decided as for a single centre
              const double xc = (double)(x0 + tx + 8 * c) - ic;
              const double yc = (double)(y0 + ty + 4 * b) - ic;
              float vv[S];
#pragma unroll
              for (int ks = 0; ks < S; ++ks) {
                const int sh = ks * gsp;
                const float dl = q - (p.qlo - (float)sh), dr = q - (p.qmax - (float)sh);
                bool in = (dl >= 0.f) && (dr <= 0.f);
                int jk = j;
                if (fabsf(dl) < kEdgeTol || fabsf(dr) < kEdgeTol) {
                  const double pe = __dadd_rn(__dadd_rn(__dmul_rn(xc, p.c64), __dmul_rn(yc, p.s64)),
                                              ctr + (double)sh);
                  in = (pe >= 0.0) && (pe <= (double)(ncol - 1));
                  jk = max(j, p.j0 - sh - kHalf);
                }
                const float4 pr = reinterpret_cast<const float4 *>(w)[(ks >> 1) * kWin + jk];
                vv[ks] = in ? fmaf((ks & 1) ? pr.w : pr.z, q, (ks & 1) ? pr.y : pr.x) : 0.f;
              }
#pragma unroll
              for (int g = 0; g < S / 2; ++g) {
                unsigned long long acc = acc2[b][c][g];
                asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc) : "l"(pack2(vv[2 * g], vv[2 * g + 1])));
                acc2[b][c][g] = acc;
              }
              continue;
            }
            if constexpr (kChecked) {
              const float dl = q - p.qlo, dr = q - p.qmax;
              inr = (dl >= 0.f) && (dr <= 0.f);
              if (fabsf(dl) < kEdgeTol || fabsf(dr) < kEdgeTol) {
                // same expression and rounding order as the reference's
                // (x - ic) cos + (y - ic) sin + center, in FP64
                const double xc = (double)(x0 + tx + 8 * c) - ic;
                const double yc = (double)(y0 + ty + 4 * b) - ic;
                const double pe =
                    __dadd_rn(__dadd_rn(__dmul_rn(xc, p.c64), __dmul_rn(yc, p.s64)), ctr);
                inr = (pe >= 0.0) && (pe <= (double)(ncol - 1));
                moved = j < p.j0 - kHalf;
                j = max(j, p.j0 - kHalf);
              }
            }
            if constexpr (K::kHalfPairs) {
              // fraction of q in its bin, then v + D f on two slices at once
              const float f = moved ? q - (float)j : q - __fsub_rn(tq, kMagic);
              const unsigned long long F = pack2(f, f);
              const uint2 *w2 = reinterpret_cast<const uint2 *>(w) + j;
#pragma unroll
              for (int g = 0; g < S / 2; ++g) {
                uint2 pw = w2[g * kWin];
                if constexpr (kChecked) {
                  if (!inr) pw = make_uint2(0u, 0u);
                }
                float v0, v1, d0, d1;
                atb::unpack_pair<T>(pw.x, v0, v1);
                atb::unpack_pair<T>(pw.y, d0, d1);
                fma_acc2(acc2[b][c][g], pack2(v0, v1), pack2(d0, d1), F);
              }
            } else if constexpr (S == 1) {
              const float2 pr = reinterpret_cast<const float2 *>(w)[j];
              float v = fmaf(pr.y, q, pr.x);
              if constexpr (kChecked) v = inr ? v : 0.f;
              if (kPerAngleKahan) kahan_add(sum[b][c][0], comp[b][c][0], v);
              else accf[b][c] += v;
            } else {
              const unsigned long long Q = pack2(q, q);
              const float4 *w4 = reinterpret_cast<const float4 *>(w) + j;
#pragma unroll
              for (int g = 0; g < S / 2; ++g) {
                float4 pr = w4[g * kWin];
                if constexpr (kChecked) {
                  if (!inr) pr = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                fma_acc2(acc2[b][c][g], pack2(pr.x, pr.y), pack2(pr.z, pr.w), Q);
              }
            }
          }
        }
      };
      if (flag & 2) body(std::true_type{});
      else body(std::false_type{});
    }
    // fold this chunk's partials into the compensated totals in TMEM
    if constexpr (!kPerAngleKahan) {
      __syncwarp();
#pragma unroll
      for (int n0 = 0; n0 < kAcc; n0 += kXfer) {
        float r[2 * kXfer];
        tmem_ld<2 * kXfer>(tm + 2 * n0, r);
#pragma unroll
        for (int i = 0; i < kXfer; ++i) kahan_add(r[2 * i], r[2 * i + 1], partial(n0 + i));
        tmem_st<2 * kXfer>(tm + 2 * n0, r);
      }
#pragma unroll
      for (int b = 0; b < PY; ++b)
#pragma unroll
        for (int c = 0; c < PX; ++c) {
          accf[b][c] = 0.f;
#pragma unroll
          for (int g = 0; g < NP; ++g) acc2[b][c][g] = 0ull;
        }
    }

    // chunk k + 1: its windows, k + 2's parameters, k + 1's pairs
    if (k + 1 < nchunk) {
      late = false;
      if (use_tma) {
        late = !mbar_wait(&raw_bar, (unsigned)((k + 1) & 1), a.wait_polls);
      } else {
        cp_async_wait_all();
        __syncthreads();  // every thread's copies landed
      }
      if (k + 2 < nchunk) params(k + 2, (k + 2) % 3);
      make_pairs(k + 1, (k + 1) % 3, (k + 1) & 1);
      if (__syncthreads_or(late)) {  // pairs(k + 1), params(k + 2) visible; raw free
        pending = k + 1;
        stalled = true;
        break;
      }
      if (k + 2 < nchunk) issue_raw(k + 2, (k + 2) % 3);
    }
  }
  if (stalled) {  // CTA-uniform; only TMA waits run out
    // a window load never completed: record it, give that copy one more
    // bounded wait, and leave without writing this tile
    if (tid == 0) atomicOr(&g_bp_status, 1);
    mbar_wait(&raw_bar, (unsigned)(pending & 1), a.wait_polls);
    return;
  }
  if constexpr (!kPerAngleKahan) {
    __syncwarp();
#pragma unroll
    for (int n0 = 0; n0 < kAcc; n0 += kXfer) {
      float r[2 * kXfer];
      tmem_ld<2 * kXfer>(tm + 2 * n0, r);
#pragma unroll
      for (int i = 0; i < kXfer; ++i) {
        const int n = n0 + i, k = n % S, c = (n / S) % PX, b = n / (S * PX);
        sum[b][c][k] = r[2 * i];
        comp[b][c][k] = r[2 * i + 1];
      }
    }
  }

  // epilogue: compensated total, circle mask, scale, store
  const int cm = ncol / 2;
#pragma unroll
  for (int b = 0; b < PY; ++b) {
    const int y = y0 + ty + 4 * b;
#pragma unroll
    for (int c = 0; c < PX; ++c) {
      const int x = x0 + tx + 8 * c;
      if (x < ncol && y < ncol) {
        bool keep = true;
        if (a.mask_r2 >= 0.0) {
          const long long dx = x - cm, dy = y - cm;
          keep = (double)(dx * dx + dy * dy) <= a.mask_r2;
        }
#pragma unroll
        for (int k = 0; k < S; ++k) {
          if (k < nsl) {
            const float v = keep ? __fsub_rn(sum[b][c][k], comp[b][c][k]) * a.scale : 0.f;
            a.out[y * a.ors + (slice0 + k) * a.oss + x] = v;
          }
        }
      }
    }
  }
}

template <typename T, int S, bool kPerAngleKahan, int V, bool kGroup = false>
__global__ void __launch_bounds__(BPCfg<T, S, V>::kThreads, BPCfg<T, S, V>::kMinBlocks)
    bp_kernel(BPArgs a, const __grid_constant__ CUtensorMap tmap) {
  using K = BPCfg<T, S, V>;
  extern __shared__ __align__(16) unsigned char smem[];
  if constexpr (kPerAngleKahan) {
    bp_tile<T, S, true, V, kGroup>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem, 0u, &tmap);
  } else {
    __shared__ uint32_t tmem_slot;
    const uint32_t tmem = tmem_alloc_cta<K::kTmemCols>(&tmem_slot);
    bp_tile<T, S, false, V, kGroup>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem, tmem, &tmap);
    tmem_free_cta<K::kTmemCols>(tmem);
  }
}

// Persistent back-projection of a batch of single-slice items of uneven
// shapes: every CTA pulls work units (item, tile) from counter[0] until the
// list is exhausted; the last CTA to leave resets counter[0] and counter[1]
// to zero, so the next launch (or graph replay) starts from a clean state.
template <typename T, int V>
__global__ void __launch_bounds__(BPCfg<T, 1, V>::kThreads, BPCfg<T, 1, V>::kMinBlocks)
    bp_batch_kernel(const atb_bp_item *items, const int *units, int nunits, int *counter) {
  using K = BPCfg<T, 1, V>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int unit_s;
  __shared__ uint32_t tmem_slot;
  const uint32_t tmem = tmem_alloc_cta<K::kTmemCols>(&tmem_slot);
  for (;;) {
    __syncthreads();  // the previous unit is done with unit_s
    if (threadIdx.x == 0) unit_s = atomicAdd(counter, 1);
    __syncthreads();
    const int u = unit_s;
    if (u >= nunits) break;
    const unsigned code = (unsigned)units[u];
    const atb_bp_item it = items[code >> 16];
    const int tile = (int)(code & 0xffffu);
    BPArgs a;
    a.sino = it.sino; a.srs = it.sino_row_stride; a.sss = 0;
    a.nrow = it.nrow; a.nslice = 1; a.ncol = it.ncol; a.slice_base = 0;
    a.trig = reinterpret_cast<const double2 *>(it.trig);
    a.center = it.center; a.edge_pad = it.edge_pad; a.mask_r2 = it.mask_r2; a.scale = it.scale;
    a.out = it.out; a.ors = it.out_row_stride; a.oss = 0;
    a.slope = 0;
    a.wait_polls = kWaitPolls;
    a.inject = 0;
    a.vec16 = sizeof(T) == 4 && (reinterpret_cast<uintptr_t>(it.sino) % 16) == 0 &&
              it.sino_row_stride % 4 == 0 && it.ncol % 4 == 0;
    a.tma = 0;
    a.spacing = 0;
    const int tiles_x = (it.ncol + K::TX - 1) / K::TX;
    bp_tile<T, 1, false, V>(a, tile % tiles_x, tile / tiles_x, 0, smem, tmem, nullptr);
  }
  tmem_free_cta<K::kTmemCols>(tmem);
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counter + 1, 1) == (int)gridDim.x - 1) {
      atomicExch(counter, 0);
      atomicExch(counter + 1, 0);
      __threadfence();
    }
  }
}

template <typename T> constexpr CUtensorMapDataType tma_type() {
  return std::is_same<T, float>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
         : std::is_same<T, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                          : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}

// cuTensorMapEncodeTiled from the driver, fetched once; null if unavailable
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The [nrow][nslice][ncol] sinogram array as a TMA tensor (bins, slices,
// angles) whose box is one angle's windows of S slices; false when the
// layout does not allow it (the kernel then stages with cp.async).
template <typename T, int S, int V, bool kGroup>
bool make_window_map(const BPArgs &a, CUtensorMap *map) {
  using K = BPCfg<T, S, V>;
  auto encode = tensor_map_encoder();
  if (!encode || !a.vec16) return false;
  const cuuint64_t es = sizeof(T);
  // vec16: 16-byte aligned base and strides; a single row per angle (one
  // slice, or a centre group's one sinogram) takes the row length as its
  // (unused) slice stride
  const bool one_row = kGroup || a.nslice == 1;
  const cuuint64_t dims[3] = {(cuuint64_t)a.ncol, one_row ? 1u : (cuuint64_t)a.nslice, (cuuint64_t)a.nrow};
  const cuuint64_t strides[2] = {one_row ? (cuuint64_t)a.ncol * es : (cuuint64_t)a.sss * es,
                                 (cuuint64_t)a.srs * es};
  // a centre group stages one row segment per angle
  const cuuint32_t box[3] = {
      (cuuint32_t)(kGroup ? group_segment(K::kWin, S, a.spacing, K::kVecElems) : K::kRaw),
      kGroup ? 1u : (cuuint32_t)S, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  if (strides[0] % 16 || strides[1] % 16 || strides[0] == 0 || strides[1] == 0) return false;
  return encode(map, tma_type<T>(), 3, const_cast<void *>(a.sino), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int S, bool kPerAngleKahan, int V = 0, bool kGroup = false>
int launch_bp(BPArgs a, int nslices, cudaStream_t st) {
  using K = BPCfg<T, S, V>;
  auto fn = bp_kernel<T, S, kPerAngleKahan, V, kGroup>;
  const int rc = atb::ensure_smem(fn, K::kSmem, "atb_backproject", K::kThreads, kPerAngleKahan ? 0 : K::kTmemCols);
  if (rc != ATB_OK) return rc;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  // TMA staging for 2- and 4-slice CTAs (a 4-slice stack of 2560 x 1801
  // measured 4 % faster); single-slice windows are small copies that TMA
  // does not speed up, so they keep cp.async
  a.tma = a.tma && S >= 2 && make_window_map<T, S, V, kGroup>(a, &map);
  dim3 grid((a.ncol + K::TX - 1) / K::TX, (a.ncol + K::TY - 1) / K::TY, (nslices + S - 1) / S);
  fn<<<grid, K::kThreads, K::kSmem, st>>>(a, map);
  return atb::check_launch("atb_backproject");
}

template <typename T>
int dispatch(BPArgs a, int per_angle_kahan, int variant, cudaStream_t st) {
  if (per_angle_kahan) return launch_bp<T, 1, true>(a, a.nslice, st);
  if (a.nslice == 1 && variant == 1) return launch_bp<T, 1, false, 1>(a, 1, st);
  // four slices per CTA for the bulk of a stack, then the remainder
  const int n4 = (a.nslice / 4) * 4;
  int rc = ATB_OK;
  if (n4 > 0) rc = launch_bp<T, 4, false>(a, n4, st);
  if (rc != ATB_OK) return rc;
  const int rem = a.nslice - n4;
  if (rem == 0) return ATB_OK;
  a.slice_base = n4;
  if (rem >= 2) {
    rc = launch_bp<T, 2, false>(a, 2, st);
    if (rc != ATB_OK || rem == 2) return rc;
    a.slice_base = n4 + 2;
  }
  if (variant == 1) return launch_bp<T, 1, false, 1>(a, 1, st);
  return launch_bp<T, 1, false>(a, 1, st);
}

}  // namespace

extern "C" int atb_backproject(const void *sino, int sino_dtype, int64_t sino_row_stride, int64_t sino_slice_stride,
                               int nrow, int nslice, int ncol, const double *trig, double center, int edge_pad,
                               double mask_r2, float scale, float *out, int64_t out_row_stride,
                               int64_t out_slice_stride, int flags, void *stream) {
  if (!sino || !trig || !out) return atb::fail(ATB_EINVAL, "atb_backproject: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1)
    return atb::fail(ATB_EINVAL, "atb_backproject: bad shape nrow=%d nslice=%d ncol=%d", nrow, nslice, ncol);
  if (nslice > 4 * 65535) return atb::fail(ATB_ERANGE, "atb_backproject: nslice=%d too large", nslice);
  if (ncol > (1 << 20)) return atb::fail(ATB_ERANGE, "atb_backproject: ncol=%d too large", ncol);
  if (!(center >= 0.0) || center >= (double)ncol)
    return atb::fail(ATB_EINVAL, "atb_backproject: center %g outside [0, %d)", center, ncol);
  BPArgs a;
  a.sino = sino; a.srs = sino_row_stride; a.sss = sino_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol; a.slice_base = 0;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.center = center; a.edge_pad = edge_pad ? 1 : 0; a.mask_r2 = mask_r2; a.scale = scale;
  a.out = out; a.ors = out_row_stride; a.oss = out_slice_stride;
  a.slope = (flags >> 1) & 1;
  a.tma = !((flags >> 4) & 1);
  // bit 5 (tests): make the first CTA's first staging wait run out, with
  // every copy complete, after a short limit
  a.inject = (flags >> 5) & 1;
  a.wait_polls = a.inject ? 4096 : kWaitPolls;
  a.spacing = 0;
  {
    const int ve = sino_dtype == ATB_F32 ? 4 : 8;  // elements per 16-byte vector
    a.vec16 = (reinterpret_cast<uintptr_t>(sino) % 16) == 0 && sino_row_stride % ve == 0 &&
              sino_slice_stride % ve == 0 && ncol % ve == 0;
  }
  cudaStream_t st = atb::as_stream(stream);
  const int pak = flags & 1;
  const int variant = (flags >> 2) & 3;
  if (variant > 1) return atb::fail(ATB_EINVAL, "atb_backproject: unknown tile variant %d", variant);
  switch (sino_dtype) {
    case ATB_F32: return dispatch<float>(a, pak, variant, st);
    case ATB_F16: return dispatch<__half>(a, pak, variant, st);
    case ATB_BF16: return dispatch<__nv_bfloat16>(a, pak, variant, st);
    default: return atb::fail(ATB_EINVAL, "atb_backproject: unknown sino_dtype %d", sino_dtype);
  }
}

extern "C" int atb_backproject_status(int reset) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_bp_status, sizeof(int)) != cudaSuccess)
    return atb::fail(ATB_ECUDA, "atb_backproject_status: %s", cudaGetErrorString(cudaGetLastError()));
  if (reset && v) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_bp_status, &zero, sizeof(int)) != cudaSuccess)
      return atb::fail(ATB_ECUDA, "atb_backproject_status: %s", cudaGetErrorString(cudaGetLastError()));
  }
  return v;
}

extern "C" int atb_backproject_centers(const float *sino, int64_t sino_row_stride, int nrow, int ncol,
                                       const double *trig, double center, int spacing, int ncenter, int edge_pad,
                                       double mask_r2, float scale, float *out, int64_t out_row_stride,
                                       int64_t out_center_stride, int flags, void *stream) {
  if (!sino || !trig || !out) return atb::fail(ATB_EINVAL, "atb_backproject_centers: null pointer");
  if (nrow < 1 || ncol < 1 || ncenter < 1)
    return atb::fail(ATB_EINVAL, "atb_backproject_centers: bad shape nrow=%d ncol=%d ncenter=%d", nrow, ncol,
                     ncenter);
  if (ncenter > 4 * 65535) return atb::fail(ATB_ERANGE, "atb_backproject_centers: ncenter=%d too large", ncenter);
  if (ncol > (1 << 20)) return atb::fail(ATB_ERANGE, "atb_backproject_centers: ncol=%d too large", ncol);
  // the staged row segment of a 4-centre CTA must fit its slot and a TMA box
  using K4 = BPCfg<float, 4, 0>;
  using K1 = BPCfg<float, 1, 0>;
  if (spacing < 1 || group_segment(K4::kWin, 4, spacing, 4) > 256 ||
      group_segment(K4::kWin, 4, spacing, 4) > K4::kRawSlot ||
      group_segment(BPCfg<float, 2, 0>::kWin, 2, spacing, 4) > BPCfg<float, 2, 0>::kRawSlot ||
      group_segment(K1::kWin, 1, spacing, 4) > K1::kRawSlot)
    return atb::fail(ATB_ERANGE, "atb_backproject_centers: spacing=%d outside [1, 56]", spacing);
  const double last = center + (double)(ncenter - 1) * (double)spacing;
  if (!(center >= 0.0) || last >= (double)ncol)
    return atb::fail(ATB_EINVAL, "atb_backproject_centers: centres %g..%g outside [0, %d)", center, last, ncol);
  BPArgs a;
  a.sino = sino; a.srs = sino_row_stride; a.sss = 0;
  a.nrow = nrow; a.nslice = ncenter; a.ncol = ncol; a.slice_base = 0;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.center = center; a.edge_pad = edge_pad ? 1 : 0; a.mask_r2 = mask_r2; a.scale = scale;
  a.out = out; a.ors = out_row_stride; a.oss = out_center_stride;
  a.slope = 0;
  a.tma = !((flags >> 4) & 1);
  a.inject = 0;
  a.wait_polls = kWaitPolls;
  a.spacing = spacing;
  a.vec16 = (reinterpret_cast<uintptr_t>(sino) % 16) == 0 && sino_row_stride % 4 == 0 && ncol % 4 == 0;
  cudaStream_t st = atb::as_stream(stream);
  // four centres per CTA, then the remainder
  const int n4 = (ncenter / 4) * 4;
  int rc = ATB_OK;
  if (n4 > 0) rc = launch_bp<float, 4, false, 0, true>(a, n4, st);
  if (rc != ATB_OK) return rc;
  const int rem = ncenter - n4;
  if (rem == 0) return ATB_OK;
  a.slice_base = n4;
  if (rem >= 2) {
    rc = launch_bp<float, 2, false, 0, true>(a, 2, st);
    if (rc != ATB_OK || rem == 2) return rc;
    a.slice_base = n4 + 2;
  }
  return launch_bp<float, 1, false, 0, true>(a, 1, st);
}

namespace {
int sm_count() {
  static int cache[64] = {0};
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev]) return cache[dev];
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  cache[dev] = n;
  return n;
}
constexpr int kBatchTile = 64;  // tile edge of single-slice variant 0
inline int batch_tile(int variant) { return variant == 1 ? 32 : 64; }
}  // namespace

extern "C" int atb_bp_batch_plan(const atb_bp_item *items, int nitems, int *units, int capacity, int variant) {
  if (!items || nitems < 1) return atb::fail(ATB_EINVAL, "atb_bp_batch_plan: no items");
  if (nitems > 65536) return atb::fail(ATB_ERANGE, "atb_bp_batch_plan: nitems=%d > 65536", nitems);
  if (variant < 0 || variant > 1) return atb::fail(ATB_EINVAL, "atb_bp_batch_plan: unknown tile variant %d", variant);
  const int tile = batch_tile(variant);
  long long total = 0;
  for (int b = 0; b < nitems; ++b) {
    const atb_bp_item &it = items[b];
    if (it.nrow < 1 || it.ncol < 1) return atb::fail(ATB_EINVAL, "atb_bp_batch_plan: item %d bad shape", b);
    const long long t = (long long)((it.ncol + tile - 1) / tile) * ((it.ncol + tile - 1) / tile);
    if (t > 65536)
      return atb::fail(ATB_ERANGE, "atb_bp_batch_plan: item %d has ncol=%d > %d", b, it.ncol, 256 * tile);
    total += t;
  }
  if (!units) return (int)total;  // size query
  if (total > capacity) return atb::fail(ATB_ERANGE, "atb_bp_batch_plan: %lld units > capacity %d", total, capacity);
  // longest-processing-time order: items by angle count, largest first
  // (every unit of an item costs nrow angle passes over one tile)
  int *order = new int[nitems];
  for (int b = 0; b < nitems; ++b) order[b] = b;
  for (int x = 1; x < nitems; ++x) {  // stable insertion sort, nitems is small
    const int v = order[x];
    int y = x - 1;
    while (y >= 0 && items[order[y]].nrow < items[v].nrow) { order[y + 1] = order[y]; --y; }
    order[y + 1] = v;
  }
  int n = 0;
  for (int q = 0; q < nitems; ++q) {
    const int b = order[q];
    const int tx = (items[b].ncol + tile - 1) / tile;
    for (int t = 0; t < tx * tx; ++t) units[n++] = (int)(((unsigned)b << 16) | (unsigned)t);
  }
  delete[] order;
  return n;
}

namespace {
template <int V>
int launch_batch(const atb_bp_item *items, int nitems, const int *units, int nunits, int *counter, int max_ctas,
                 cudaStream_t st) {
  using K = BPCfg<float, 1, V>;
  const int rc = atb::ensure_smem(bp_batch_kernel<float, V>, K::kSmem, "atb_backproject_batch", K::kThreads, K::kTmemCols);
  if (rc != ATB_OK) return rc;
  int grid = K::kMinBlocks * sm_count();
  if (max_ctas > 0 && max_ctas < grid) grid = max_ctas;
  if (grid > nunits) grid = nunits;
  bp_batch_kernel<float, V><<<grid, K::kThreads, K::kSmem, st>>>(items, units, nunits, counter);
  return atb::check_launch("atb_backproject_batch");
}
}  // namespace

extern "C" int atb_backproject_batch(const atb_bp_item *items, int nitems, const int *units, int nunits,
                                     int *counter, int max_ctas, int variant, void *stream) {
  if (!items || !units || !counter) return atb::fail(ATB_EINVAL, "atb_backproject_batch: null pointer");
  if (nitems < 1 || nunits < 1) return atb::fail(ATB_EINVAL, "atb_backproject_batch: empty batch");
  static_assert(BPCfg<float, 1, 0>::TX == kBatchTile && BPCfg<float, 1, 0>::TY == kBatchTile, "square tiles");
  static_assert(BPCfg<float, 1, 1>::TX == 32 && BPCfg<float, 1, 1>::TY == 32, "square tiles");
  cudaStream_t st = atb::as_stream(stream);
  switch (variant) {
    case 0: return launch_batch<0>(items, nitems, units, nunits, counter, max_ctas, st);
    case 1: return launch_batch<1>(items, nitems, units, nunits, counter, max_ctas, st);
    default: return atb::fail(ATB_EINVAL, "atb_backproject_batch: unknown tile variant %d", variant);
  }
}

// ---------------------------------------------------------------------------
// Batched back-projection for callers that cannot allocate device memory.
//
// Some callers hold device buffers for their inputs and outputs but may not
// call cudaMalloc themselves: a plugin inside an application whose memory
// pool must account for every device byte, a latency-bound loop that cannot
// afford cudaMalloc's implicit synchronisation, or a foreign-language caller
// that is handed device pointers but has no CUDA runtime to allocate with.
// atb_backproject_batch needs three small device scratch buffers from its
// caller (item table, work list, counter).  The entry point below keeps them
// instead in one file-scope __device__ array of fixed size, which every GPU
// that loads this library holds until the process exits.
//
// Nothing of the call stays in host memory: the item table travels to the
// device inside the parameters of small upload launches (each launch's
// parameters are copied when it is enqueued), and the work list is built on
// the device from that table, in the same longest-processing-time order as
// atb_bp_batch_plan.  So the caller may reuse or free its host table as soon
// as the call returns, and the call never waits for earlier work on the
// stream (no copy from pageable host memory).
namespace {

constexpr int kNoAllocMaxItems = 4096;
constexpr int kNoAllocMaxUnits = 1 << 20;
constexpr size_t kNoAllocItemsOffset = 256;  // the counter pair sits first
constexpr size_t kNoAllocUnitsOffset =
    kNoAllocItemsOffset + ((sizeof(atb_bp_item) * kNoAllocMaxItems + 255) / 256) * 256;
constexpr size_t kNoAllocBytes = kNoAllocUnitsOffset + sizeof(int) * (size_t)kNoAllocMaxUnits;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// items per upload launch: the chunk stays inside the 32764-byte kernel
// parameter limit of sm_70 and later devices (CUDA 12.1 and later)
constexpr int kNoAllocChunk = 440;
struct NoAllocChunk {
  int first, count;
  atb_bp_item items[kNoAllocChunk];
};
static_assert(sizeof(NoAllocChunk) + sizeof(void *) <= 32764, "upload chunk exceeds the kernel parameter limit");

__global__ void __launch_bounds__(256) noalloc_upload_kernel(const __grid_constant__ NoAllocChunk c,
                                                             atb_bp_item *dst) {
  for (int k = threadIdx.x; k < c.count; k += blockDim.x) dst[c.first + k] = c.items[k];
}

// Work list of the uploaded table: units[o_r + t] = item << 16 | t for the
// item of rank r in (angle count descending, index ascending) order, o_r the
// sum of the tile counts of the ranks before r; also zeroes the counter pair
// (the array keeps the previous call's contents).  One CTA.
__global__ void __launch_bounds__(1024) noalloc_plan_kernel(const atb_bp_item *items, int nitems, int *units,
                                                            int *counter) {
  __shared__ int key[kNoAllocMaxItems];   // angle counts, then tile counts by rank, then offsets
  __shared__ int item_at[kNoAllocMaxItems];
  __shared__ int warp_sum[32];
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) {
    counter[0] = 0;
    counter[1] = 0;
  }
  for (int b = tid; b < nitems; b += nt) key[b] = items[b].nrow;
  __syncthreads();
  for (int b = tid; b < nitems; b += nt) {  // stable rank, largest angle count first
    const int kb = key[b];
    int r = 0;
    for (int j = 0; j < nitems; ++j) {
      const int kj = key[j];
      r += (kj > kb) || (kj == kb && j < b);
    }
    item_at[r] = b;
  }
  __syncthreads();
  int tiles[4];
  int local = 0;
  for (int q = 0; q < 4; ++q) {  // each thread owns ranks 4 tid .. 4 tid + 3
    const int r = 4 * tid + q;
    int t = 0;
    if (r < nitems) {
      const int tx = (items[item_at[r]].ncol + kBatchTile - 1) / kBatchTile;
      t = tx * tx;
    }
    tiles[q] = t;
    local += t;
  }
  // exclusive scan of the per-thread sums over the CTA
  const int lane = tid & 31, warp = tid >> 5;
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (nt >> 5) ? warp_sum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    warp_sum[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  int off = incl - local + (warp > 0 ? warp_sum[warp - 1] : 0);
  for (int q = 0; q < 4; ++q) {
    const int r = 4 * tid + q;
    if (r < nitems) key[r] = off;
    off += tiles[q];
  }
  __syncthreads();
  for (int r = 0; r < nitems; ++r) {
    const int b = item_at[r];
    const int tx = (items[b].ncol + kBatchTile - 1) / kBatchTile;
    const int o = key[r];
    for (int t = tid; t < tx * tx; t += nt) units[o + t] = (int)(((unsigned)b << 16) | (unsigned)t);
  }
}

// per-device address of g_noalloc_scratch, looked up once per device, and
// the host-side upload chunk (static rather than on the caller's stack);
// both guarded by g_noalloc_mu
unsigned char *g_noalloc_dev[64] = {nullptr};
NoAllocChunk g_noalloc_chunk;
std::mutex g_noalloc_mu;

}  // namespace

extern "C" int atb_backproject_batch_noalloc(const atb_bp_item *items, int nitems, int max_ctas, void *stream) {
  if (!items) return atb::fail(ATB_EINVAL, "atb_backproject_batch_noalloc: null item table");
  if (nitems < 1) return atb::fail(ATB_EINVAL, "atb_backproject_batch_noalloc: empty batch");
  if (nitems > kNoAllocMaxItems)
    return atb::fail(ATB_ERANGE, "atb_backproject_batch_noalloc: nitems=%d exceeds the fixed limit of %d items",
                     nitems, kNoAllocMaxItems);
  long long nunits = 0;
  for (int b = 0; b < nitems; ++b) {
    const atb_bp_item &it = items[b];
    if (!it.sino || !it.trig || !it.out || it.nrow < 1 || it.ncol < 1)
      return atb::fail(ATB_EINVAL, "atb_backproject_batch_noalloc: item %d is incomplete", b);
    if (it.ncol > 16384)
      return atb::fail(ATB_ERANGE, "atb_backproject_batch_noalloc: item %d has ncol=%d > 16384", b, it.ncol);
    const long long t = (it.ncol + kBatchTile - 1) / kBatchTile;
    nunits += t * t;
  }
  if (nunits > kNoAllocMaxUnits)
    return atb::fail(ATB_ERANGE,
                     "atb_backproject_batch_noalloc: %lld tiles of 64 x 64 exceed the fixed limit of %d",
                     nunits, kNoAllocMaxUnits);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return atb::fail(ATB_ECUDA, "atb_backproject_batch_noalloc: no usable current device");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_dev[dev]) {  // first call on this device: device address of the scratch array
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return atb::fail(ATB_ECUDA, "atb_backproject_batch_noalloc: cudaGetSymbolAddress: %s",
                       cudaGetErrorString(e));
    g_noalloc_dev[dev] = static_cast<unsigned char *>(p);
  }
  unsigned char *base = g_noalloc_dev[dev];
  int *counter = reinterpret_cast<int *>(base);
  atb_bp_item *items_dev = reinterpret_cast<atb_bp_item *>(base + kNoAllocItemsOffset);
  int *units_dev = reinterpret_cast<int *>(base + kNoAllocUnitsOffset);
  cudaStream_t st = atb::as_stream(stream);

  using K = BPCfg<float, 1, 0>;
  const int rc =
      atb::ensure_smem(bp_batch_kernel<float, 0>, K::kSmem, "atb_backproject_batch_noalloc", K::kThreads, K::kTmemCols);
  if (rc != ATB_OK) return rc;
  NoAllocChunk &chunk = g_noalloc_chunk;
  for (int first = 0; first < nitems; first += kNoAllocChunk) {
    chunk.first = first;
    chunk.count = nitems - first < kNoAllocChunk ? nitems - first : kNoAllocChunk;
    std::memcpy(chunk.items, items + first, sizeof(atb_bp_item) * (size_t)chunk.count);
    noalloc_upload_kernel<<<1, 256, 0, st>>>(chunk, items_dev);
    const int r = atb::check_launch("atb_backproject_batch_noalloc (item upload)");
    if (r != ATB_OK) return r;
  }
  noalloc_plan_kernel<<<1, 1024, 0, st>>>(items_dev, nitems, units_dev, counter);
  const int r = atb::check_launch("atb_backproject_batch_noalloc (work list)");
  if (r != ATB_OK) return r;
  int grid = 2 * sm_count();
  if (max_ctas > 0 && max_ctas < grid) grid = max_ctas;
  if (grid > nunits) grid = (int)nunits;
  bp_batch_kernel<float, 0><<<grid, K::kThreads, K::kSmem, st>>>(items_dev, units_dev, (int)nunits, counter);
  return atb::check_launch("atb_backproject_batch_noalloc");
}
