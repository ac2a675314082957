// k_closure.cu - the learned vertical closure: BF16 inference of the MLP 8 -> 64 -> 64 -> 3
// on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory), fused
// with the closure's update of KQ, KM, KH.
//
// VDIF_Q in learned mode (P.closure == 1) stores, for every wet node and interior level,
// the eight network inputs transformed, standardised and rounded to BF16 (clos_feat: one
// 16-byte row, the MMA's A-operand row as it goes into shared memory), and per column
// whether the node is wet and all its inputs lie inside the training envelope (clos_env,
// from per-chunk flags of VDIF_Q's level kernel).  VDIF_Q finishes every column outside
// the envelope with MY2.5 (the per-column fallback) and leaves KQ, KM, KH of the interior
// levels of the others to the network: k_clos_count and k_clos_list compact the columns
// on the network into an ordered list, and k_closure_mlp runs the network on the rows
// (interior level, listed column) only, takes its prediction and averages with the old
// value as MY2.5 does: K = 0.5*(new + K_old) (vdif_q.F:489-491).
//
// Tile scheme: a CTA of 128 threads owns tiles of 128 rows; thread t owns row t of the
// tile and TMEM lane t.  For each layer the threads write their row's BF16 activations
// into shared memory in the canonical no-swizzle K-major layout (core matrices of 8 rows
// x 16 bytes; core (row group g, k group c) at g*SBO + c*128 bytes), one elected thread
// issues tcgen05.mma (M=128, N=64 or 16, K=16 per instruction, FP32 accumulate), commits
// to an mbarrier and waits on it while the others wait at the block barrier, and every
// thread reads its row back with tcgen05.ld, adds the bias (from shared memory) and
// applies GELU (packed FP16, gelu2_bf16).  Weights and biases are staged once per CTA.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "fvg_model.h"

namespace fvg {

namespace {

constexpr int ROWS = 128;          // rows per tile = MMA M = threads per CTA
constexpr int K1 = 16;             // layer-1 K (8 inputs padded with zeros)
constexpr int HID = 64;            // hidden width = MMA N of layers 1 and 2
constexpr int NOUT = 16;           // layer-3 N (3 outputs padded)
constexpr int CORE = 128;          // bytes of one core matrix (8 rows x 16 bytes)
// shared-memory image (bytes)
constexpr int S_W1 = 0;                           // 64 x 16 bf16, SBO 256
constexpr int S_W2 = S_W1 + HID * K1 * 2;         // 64 x 64 bf16, SBO 1024
constexpr int S_W3 = S_W2 + HID * HID * 2;        // 16 x 64 bf16, SBO 1024
constexpr int S_A1 = S_W3 + NOUT * HID * 2;         // 128 x 16 bf16, SBO 256
constexpr int S_A2 = S_A1 + ROWS * K1 * 2;        // 128 x 64 bf16, SBO 1024
constexpr int S_B = S_A2 + ROWS * HID * 2;        // biases b1, b2, b3 (64 + 64 + 16 FP32)
constexpr int S_END = S_B + (2 * HID + NOUT) * 4;
constexpr int W_IMAGE = S_A1;                     // bytes of the weight image
// TMEM columns: D1, D2 and D3 all at [0,64) -- each layer's accumulator is read out (and
// the read waited for) before the next layer's MMA is issued -- so 64 columns are
// allocated and eight CTAs fit in an SM's 512 columns.
constexpr uint32_t TMEM_COLS = 64;
constexpr int kCtasPerSm = 6;  // resident CTAs per SM the launch bounds ask for
constexpr long kSpin = 1 << 22;  // bound of every mbarrier wait

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: no swizzle, K-major, version 1.
__device__ inline uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version
  return d;                 // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4)                     // D format FP32
         | (1u << 7)                   // A format BF16
         | (1u << 10)                  // B format BF16
         | ((uint32_t)(n >> 3) << 17)  // N / 8
         | ((uint32_t)(m >> 4) << 24);  // M / 16
}

__device__ inline void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.u32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate));
}

__device__ inline void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false if it ran out.
__device__ inline bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  const uint32_t a = smem_u32(mbar);
  for (long it = 0; it < kSpin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ inline void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ inline void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ inline uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// GELU of two values, rounded to a BF16 pair: the tanh argument and 0.5*(1 + tanh) are
// formed in packed FP16 with one hardware tanh for both values (its error, about 2^-11, is
// that of the FP32 hardware tanh and far below the BF16 rounding of the result), and the
// product with z in FP32.  Half the tanh instructions and about half the arithmetic of
// two FP32 evaluations.  For |z| beyond FP16's range the argument saturates to +-inf,
// where tanh is +-1 and GELU(z) = z or 0, as in FP32.
__device__ inline uint32_t gelu2_bf16(float z0, float z1) {
  const __half2 zh = __floats2half2_rn(z0, z1);
  const __half2 z2 = __hmul2(zh, zh);
  const __half2 p = __hfma2(z2, __float2half2_rn(0.0356774081f), __float2half2_rn(0.7978845608f));
  const __half2 u = __hmul2(zh, p);
  uint32_t ui = *reinterpret_cast<const uint32_t*>(&u), ti;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(ti) : "r"(ui));
  const __half2 t = *reinterpret_cast<const __half2*>(&ti);
  const __half2 hh = __hfma2(t, __float2half2_rn(0.5f), __float2half2_rn(0.5f));
  const float2 h = __half22float2(hh);
  return pack_bf16(z0 * h.x, z1 * h.y);
}

// Row r (0..127) of an activation tile with K columns (multiple of 8): 8 values per
// 16-byte store at core (r/8, c) row r%8.
template <int K>
__device__ inline void store_row(uint8_t* tile, int sbo, int r, const float* v) {
#pragma unroll
  for (int c = 0; c < K / 8; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + (r / 8) * sbo + c * CORE + (r % 8) * 16) = q;
  }
}

// Sixteen BF16 values of row r (eight packed pairs) into core-matrix columns c8 and c8+1
// of an activation tile.
__device__ inline void store_cols16_bf16(uint8_t* tile, int sbo, int r, int c8, const uint32_t* q) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
    *reinterpret_cast<uint4*>(tile + (r / 8) * sbo + (c8 + h) * CORE + (r % 8) * 16) =
        make_uint4(q[4 * h], q[4 * h + 1], q[4 * h + 2], q[4 * h + 3]);
}

}  // namespace

// The tile pipeline shared by the closure and the standalone forward pass.  need(r): row r
// goes through the network; load(r, v) fills the 8 standardised inputs of such a row (the
// next tile's rows are fetched while the current tile runs); prefetch(r) is called while
// the last layer's MMA runs, so that the caller can fetch what store needs; store(r, o,
// true) receives the 3 network outputs (bias included).  If an mbarrier wait runs out, err
// receives 1 and every row of the block that has not been stored yet (the current tile
// and all later ones) gets store(r, nullptr, false).
template <class Load, class Store, class Need, class Prefetch>
__device__ inline void mlp_tc_tiles(const void* wimg, const float* bias, int nrows, Load load, Store store, Need need,
                                    Prefetch prefetch, int* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int t = threadIdx.x, warp = t >> 5;
  const int ntiles = (nrows + ROWS - 1) / ROWS;
  // stage the weight image (bf16, core-matrix layout) and allocate TMEM
  for (int q = t; q < W_IMAGE / 16; q += ROWS) reinterpret_cast<uint4*>(sm)[q] = reinterpret_cast<const uint4*>(wimg)[q];
  float* const sb = reinterpret_cast<float*>(sm + S_B);
  for (int q = t; q < 2 * HID + NOUT; q += ROWS) sb[q] = q < 2 * HID + 3 ? bias[q] : 0.f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tm = tmem_base;
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  const uint32_t s0 = smem_u32(sm);
  uint32_t phase = 0;
  // the biases from shared memory, four at a time
  const float4* const b1 = reinterpret_cast<const float4*>(sb);
  const float4* const b2 = reinterpret_cast<const float4*>(sb + HID);
  const float* const b3 = sb + 2 * HID;

  // this thread's row of the next tile: whether it uses the network, and its inputs
  float vn[K1];
  bool nn = false;
  auto fetch = [&](int tl) {
    const int rr = tl * ROWS + t;
#pragma unroll
    for (int f = 0; f < K1; ++f) vn[f] = 0.f;
    nn = tl < ntiles && rr < nrows && need(rr);
    if (nn) load(rr, vn);
  };
  fetch(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r = tile * ROWS + t;
    const bool live = r < nrows;
    float v[K1];
#pragma unroll
    for (int f = 0; f < K1; ++f) v[f] = vn[f];
    const bool nd = nn;
    fetch(tile + gridDim.x);
    // after a wait ran out, the rest of the block's rows are not stored
    if (abort_flag) {
      if (live) store(r, nullptr, false);
      continue;
    }
    // a tile none of whose rows uses the network skips the tensor cores
    if (!__syncthreads_or(nd)) {
      float o[16] = {};
      if (live) store(r, o, true);
      continue;
    }
    store_row<K1>(sm + S_A1, 256, t, v);
    fence_async_smem();
    fence_before();
    __syncthreads();
    for (int layer = 0; layer < 3; ++layer) {
      if (t == 0) {
        fence_after();
        if (layer == 0) {
          mma_bf16(tm + 0, sdesc(s0 + S_A1, CORE, 256), sdesc(s0 + S_W1, CORE, 256), idesc_bf16(ROWS, HID), false);
        } else {
          const uint32_t dcol = 0u;
          const uint32_t bw = layer == 1 ? S_W2 : S_W3;
          const uint32_t idesc = idesc_bf16(ROWS, layer == 1 ? HID : NOUT);
          for (int s = 0; s < HID / 16; ++s)
            mma_bf16(tm + dcol, sdesc(s0 + S_A2 + s * 2 * CORE, CORE, 1024), sdesc(s0 + bw + s * 2 * CORE, CORE, 1024),
                     idesc, s > 0);
        }
        mma_commit(&mbar);
      }
      if (layer == 2 && live && nd) prefetch(r);
      // one thread waits for the MMAs (the others wait at the barrier, issuing nothing);
      // the barrier and each thread's tcgen05 fence then order the accumulator reads
      if (t == 0 && !mbar_wait(&mbar, phase & 1)) {
        abort_flag = 1;
        atomicExch(err, 1);
      }
      phase += 1;
      __syncthreads();
      if (abort_flag) break;
      fence_after();
      if (layer < 2) {
        const float4* bb = layer == 0 ? b1 : b2;
        // sixteen accumulator columns at a time: bias, GELU, BF16 into the next layer's
        // A tile (two core-matrix columns), so that few values are live at once
#pragma unroll
        for (int c = 0; c < HID / 16; ++c) {
          float w[16];
          tmem_ld16(tm + lane_off + 16 * c, w);
          uint32_t q[8];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float4 b = bb[4 * c + j];
            q[2 * j] = gelu2_bf16(w[4 * j] + b.x, w[4 * j + 1] + b.y);
            q[2 * j + 1] = gelu2_bf16(w[4 * j + 2] + b.z, w[4 * j + 3] + b.w);
          }
          store_cols16_bf16(sm + S_A2, 1024, t, 2 * c, q);
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
      } else {
        float o[16];
        tmem_ld16(tm + lane_off + 0, o);
        fence_before();
        if (live) {
          for (int c = 0; c < 3; ++c) o[c] += b3[c];
          store(r, o, true);
        }
        __syncthreads();
      }
    }
    // the wait of this tile ran out: none of its rows was stored
    if (abort_flag && live) store(r, nullptr, false);
  }
  // After a wait ran out, one commit is still outstanding: wait for it once more (again
  // bounded) so that the MMAs writing this block's columns are done before they are freed.
  // If that wait runs out too, err holds 2 and the columns are freed regardless: a CTA
  // must release its tensor memory before it exits, and the step's result is already
  // reported as failed.
  if (abort_flag && t == 0) {
    if (!mbar_wait(&mbar, (phase + 1) & 1)) atomicExch(err, 2);  // the phase that ran out
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TMEM_COLS));
  }
}

// Ordered compaction of the columns on the network (clos_env != 0) into clos_list, in two
// passes over blocks of kListBlock nodes: per-block counts, then each block's offset (the
// sum of the counts before it) plus an exclusive scan inside the block.  Nodes stay in
// ascending order.
constexpr int kListBlock = 1024;  // nodes per block: 256 threads x 4
__device__ inline int block_exclusive_scan(int v, int* ws, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  int before = 0;
  total = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    if (w < warp) before += ws[w];
    total += ws[w];
  }
  return before + x - v;
}
__global__ void __launch_bounds__(256) k_clos_count(const Dev P) {
  __shared__ int ws[8];
  const int i0 = blockIdx.x * kListBlock + threadIdx.x * 4 + 1;
  int c = 0;
  for (int q = 0; q < 4; ++q) c += (i0 + q <= P.M && P.clos_env[i0 + q] != 0) ? 1 : 0;
  int total;
  block_exclusive_scan(c, ws, total);
  if (threadIdx.x == 0) P.clos_cnt[blockIdx.x] = total;
}
__global__ void __launch_bounds__(256) k_clos_list(const Dev P) {
  __shared__ int ws[8];
  __shared__ int base;
  if (threadIdx.x < 32) {
    int b = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += 32) b += P.clos_cnt[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
    if (threadIdx.x == 0) base = b;
  }
  const int i0 = blockIdx.x * kListBlock + threadIdx.x * 4 + 1;
  bool on[4];
  int c = 0;
  for (int q = 0; q < 4; ++q) {
    on[q] = i0 + q <= P.M && P.clos_env[i0 + q] != 0;
    c += on[q] ? 1 : 0;
  }
  int total;
  int pos = block_exclusive_scan(c, ws, total) + base;
  for (int q = 0; q < 4; ++q)
    if (on[q]) P.clos_list[1 + pos++] = i0 + q;
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) P.clos_list[0] = base + total;
}

// The closure step.  VDIF_Q has finished every column outside the envelope with MY2.5 and
// left the BF16 inputs of the others in clos_feat (row (K-2)*M + (I-1)); this kernel
// finishes the columns on the network: its rows are (level K, j-th column on the network)
// with r = (K-2)*n + j, n = clos_list[0], node I = clos_list[1 + j].  After a wait ran out
// (store with net_ok false) a row keeps its coefficients, and the step reports
// FVG_ERR_TIMEOUT.
__global__ void __launch_bounds__(ROWS, kCtasPerSm) k_closure_mlp(const Dev P, int* err) {
  const int nnet = P.clos_list[0];
  const int nrows = nnet * (P.KBM1 - 1);
  const int* const list = P.clos_list + 1;
  const ClosNorm& nm = P.clos_norm;
  auto node_of = [&](int r) { return list[r % nnet]; };
  auto load = [&](int r, float* v) {
    const uint4 w = P.clos_feat[(size_t)(r / nnet) * P.M + (node_of(r) - 1)];
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u[j]));
      v[2 * j] = f.x;
      v[2 * j + 1] = f.y;
    }
  };
  double kold[3] = {0.0, 0.0, 0.0};  // KQ, KM, KH of the row, fetched during the last MMA
  auto prefetch = [&](int r) {
    const size_t q = N3(P, node_of(r), r / nnet + 2);
    kold[0] = P.kq[q];
    kold[1] = P.km[q];
    kold[2] = P.kh[q];
  };
  auto store = [&](int r, const float* o, bool net_ok) {
    const int k = r / nnet + 2, i = node_of(r);
    if (!net_ok) return;
    const size_t q = N3(P, i, k);
    double nw[3];
    for (int c = 0; c < 3; ++c) {
      float y = o[c] * nm.tstd[c] + nm.tmean[c];
      nw[c] = (double)expf(y) - (double)nm.teps;
      if (nw[c] < 0.0) nw[c] = 0.0;
    }
    P.kq[q] = 0.5 * (nw[0] + kold[0]);
    P.km[q] = 0.5 * (nw[1] + kold[1]);
    P.kh[q] = 0.5 * (nw[2] + kold[2]);
  };
  auto need = [](int) { return true; };
  mlp_tc_tiles(P.clos_w, P.clos_b, nrows, load, store, need, prefetch, err);
}

// Standalone BF16 forward pass on standardised inputs x [n][8] -> out [n][3].
__global__ void __launch_bounds__(ROWS, kCtasPerSm) k_mlp_tc_forward(const void* wimg, const float* bias, const float* x,
                                                            int n, float* out, int* err) {
  auto load = [&](int r, float* v) {
#pragma unroll
    for (int f = 0; f < CLOS_IN; ++f) v[f] = x[(size_t)r * CLOS_IN + f];
  };
  auto store = [&](int r, const float* o, bool net_ok) {
    for (int c = 0; c < 3; ++c) out[(size_t)r * 3 + c] = net_ok ? o[c] : __int_as_float(0x7fc00000);
  };
  auto need = [](int) { return true; };
  auto prefetch = [](int) {};
  mlp_tc_tiles(wimg, bias, n, load, store, need, prefetch, err);
}

// VDIF_Q's averaging of shallow columns (vdif_q.F:494-512), after the per-level update of
// KQ, KM, KH (MY2.5 or the network).
__global__ void k_closure_shallow(const Dev P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M || P.h[i] > P.static_ssh_adj) return;
  const int KBM1 = P.KBM1;
  double kqt = 0.0, kmt = 0.0, kht = 0.0;
  for (int k = 2; k <= KBM1; ++k) { kqt = kqt + P.kq[N3(P, i, k)]; kmt = kmt + P.km[N3(P, i, k)]; kht = kht + P.kh[N3(P, i, k)]; }
  kqt = kqt / (double)(KBM1 - 1);
  kmt = kmt / (double)(KBM1 - 1);
  kht = kht / (double)(KBM1 - 1);
  for (int k = 2; k <= KBM1; ++k) { P.kq[N3(P, i, k)] = kqt; P.km[N3(P, i, k)] = kmt; P.kh[N3(P, i, k)] = kht; }
}

size_t closure_smem_bytes() { return (size_t)S_END; }
int closure_ctas_per_sm() { return kCtasPerSm; }
size_t closure_weight_image_bytes() { return (size_t)W_IMAGE; }

void launch_vdif_q_shallow(const Dev& P, cudaStream_t s) {
  k_closure_shallow<<<(P.M + 127) / 128, 128, 0, s>>>(P);
}

void launch_closure(const Dev& P, cudaStream_t s, int* err, int grid) {
  const int nb = P.M / kListBlock + 1;
  k_clos_count<<<nb, 256, 0, s>>>(P);
  k_clos_list<<<nb, 256, 0, s>>>(P);
  k_closure_mlp<<<grid, ROWS, S_END, s>>>(P, err);
  k_closure_shallow<<<(P.M + 127) / 128, 128, 0, s>>>(P);
}

int closure_setup_attrs() {
  if (cudaFuncSetAttribute(k_closure_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S_END) != cudaSuccess)
    return 1;
  if (cudaFuncSetAttribute(k_mlp_tc_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S_END) != cudaSuccess)
    return 1;
  return 0;
}

void launch_mlp_tc_forward(const void* wimg, const float* bias, const float* x, int n, float* out, int* err, int grid,
                           cudaStream_t s) {
  k_mlp_tc_forward<<<grid, ROWS, S_END, s>>>(wimg, bias, x, n, out, err);
}

// Round to nearest even BF16: the IEEE binary32 bits with the low 16 discarded, rounding
// half to even on the discarded part.
static uint16_t bf16_rne(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16 | ((u & 0xFFFF) ? 0x40 : 0));
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// Element (n, k) of a K-major matrix in core matrices of 8 rows x 8 elements, core (g, c)
// at g*sbo + c*128 bytes.
static void put_core(std::vector<uint8_t>& img, size_t base, int sbo, int n, int k, uint16_t v) {
  size_t off = base + (size_t)(n / 8) * sbo + (size_t)(k / 8) * 128 + (size_t)(n % 8) * 16 + (size_t)(k % 8) * 2;
  img[off] = (uint8_t)(v & 0xFF);
  img[off + 1] = (uint8_t)(v >> 8);
}

void closure_weight_image(const float* params, std::vector<uint8_t>& img, std::vector<float>& bias) {
  const float* W1 = params;
  const float* B1 = W1 + 64 * 8;
  const float* W2 = B1 + 64;
  const float* B2 = W2 + 64 * 64;
  const float* W3 = B2 + 64;
  const float* B3 = W3 + 3 * 64;
  img.assign(W_IMAGE, 0);
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 8; ++k) put_core(img, S_W1, 256, n, k, bf16_rne(W1[n * 8 + k]));
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 64; ++k) put_core(img, S_W2, 1024, n, k, bf16_rne(W2[n * 64 + k]));
  for (int n = 0; n < 3; ++n)
    for (int k = 0; k < 64; ++k) put_core(img, S_W3, 1024, n, k, bf16_rne(W3[n * 64 + k]));
  bias.assign(2 * HID + NOUT, 0.f);
  for (int j = 0; j < 64; ++j) { bias[j] = B1[j]; bias[64 + j] = B2[j]; }
  for (int j = 0; j < 3; ++j) bias[128 + j] = B3[j];
}

}  // namespace fvg
