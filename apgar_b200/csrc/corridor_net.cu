// The learned corridor: a 6-layer 3x3 CNN (32 channels, BF16 weights and
// activations, FP32 accumulation) over 64 x 64 coarse rasters of each net's
// window, trained on the GPU by its own forward and backward kernels.
//
// Layout.  Every net owns a 64 x 64 coarse grid (coarse cell = 2^s x 2^s
// window cells on all layers, the corridor bitmap's scale); only the top-left
// cw x ch cells lie inside the window.  Tensors are NHWC bf16 [net][66][64][C]
// (grid row y stored at y + 1); the producers write the pad row above and
// grid rows 0 .. ch with the cells outside the window as zeros ("same"
// padding at the window border), which is all an in-window output reads
// (for a window at most 31 columns wide, the convolutions write columns
// 0 .. 31 only).
//
// Layers 1-5 (3x3, 16 -> 32 then 32 -> 32, bias, ReLU) run as implicit GEMMs
// on the 5th-generation tensor cores: a tile is 128 output cells (two rows of
// one net); TMA stages its four input rows once as channel planes in shared
// memory, each of the 9 taps' A operands is a shifted descriptor into that
// stage (M = 128 cells, K = Cin, K-major, no swizzle, no im2col copy), the
// weights stay resident as the B operand (N = 32 channels), and one thread
// issues tcgen05.mma (kind::f16, bf16 x bf16 -> f32) into a 128 x 32
// tensor-memory accumulator.  Loads, MMAs and the epilogue (tcgen05.ld, one
// warp per 32 TMEM lanes: bias, ReLU, bf16 stores) are separate warp roles
// handed over by mbarriers, several tiles in flight.
// The input gradient of layers 2-5 is the same kernel run on the output
// gradient with the spatially flipped, transposed weights; its epilogue gates
// by the previous layer's ReLU.  The weight gradient is a second tcgen05 GEMM:
// D[(tap, ci)][co] = sum over cells of im2col(x)[cell][(tap, ci)] *
// dy[cell][co], with both operands MN-major (the cell index is K), so the NHWC
// rows load as 16-byte chunks; each CTA accumulates its cells in TMEM and adds
// its partial sums to the FP32 gradient once.
//
// The head (3x3, 32 -> 1, FP32 weights), the loss, the bias gradients, Adam
// and the corridor extraction are small and run on the CUDA cores.
//
// Every mbarrier wait (TMA loads, tensor-core completions, the hand-offs
// between warp roles) is bounded: on expiry the kernel records
// APGAR_B200_CNN_TIMEOUT in its error word, waits once more (bounded) for its
// own copies and MMAs in flight, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "apgar_b200.h"
#include "lattice_common.cuh"

namespace apgar_b200 {
namespace {

constexpr int kGrid = 64;          // coarse cells per side
constexpr int kCells = kGrid * kGrid;
constexpr int kCin0 = 16;          // raster channels
constexpr int kCh = 32;            // hidden channels
constexpr uint32_t kWaitLimit = 1u << 22;

// ----------------------------- tcgen05 helpers -----------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension and
// stride-dimension byte offsets (16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: bf16 A and B, f32 accumulator, M x N,
// K-major (0) or MN-major (1) operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn) << 15) |
         (static_cast<uint32_t>(b_mn) << 16) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the barrier phase with parity `phase`; true when it completed.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Warp 0 allocates `cols` TMEM columns; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// 32 consecutive f32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t dims_w(uint32_t d) { return d & 0xFFu; }
__device__ __forceinline__ uint32_t dims_h(uint32_t d) { return (d >> 8) & 0xFFu; }

// Logits, labels: [net][64][64].
__device__ __forceinline__ size_t grid_cell(uint32_t net, int y, int x) {
  return (static_cast<size_t>(net) * kGrid + static_cast<size_t>(y)) * kGrid + static_cast<size_t>(x);
}

// Rasters, activations and their gradients: [net][66][64][c], row y stored
// at y + 1.  Rows -1 and 64 and, in rows 0 .. ch, the columns cw .. 63 hold
// zeros (the producers write them), and cw <= 63, so a 3 x 3 tap that leaves
// a row through its left or right end reads a zero or feeds an output outside
// the window; rows and columns are then plain offsets of one 64-cell pitch.
constexpr int kPadRows = kGrid + 2;
__device__ __forceinline__ size_t act_cell(uint32_t net, int y, int x) {
  return (static_cast<size_t>(net) * kPadRows + static_cast<size_t>(y + 1)) * kGrid + static_cast<size_t>(x);
}

__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 o;
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]),
                  c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
  o.x = *reinterpret_cast<uint32_t*>(&a);
  o.y = *reinterpret_cast<uint32_t*>(&b);
  o.z = *reinterpret_cast<uint32_t*>(&c);
  o.w = *reinterpret_cast<uint32_t*>(&d);
  return o;
}

__device__ __forceinline__ void unpack8(uint4 q, float* v) {
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[2 * i] = __uint_as_float(w[i] << 16);
    v[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
  }
}

// ------------------------------- rasters ----------------------------------

// One block per net: the 16 input channels of every coarse cell of rows
// -1 .. ch (the rows any in-window output reads; row ch and the columns
// cw .. 63 are zero), plus the net's coarse dims (cw | ch << 8 | s << 16).
// The blocked counts are gathered over (fine row, mask word) pairs of the
// window, every layer's word of a pair loaded together, and summed per
// coarse cell exactly (integer shared-memory atomics); a thread per coarse
// cell then forms its channels.
__global__ void __launch_bounds__(256) raster_kernel(LatticeDeviceView lat,
                                                     const apgar_b200_lattice_net* __restrict__ nets,
                                                     uint32_t count, const uint32_t* __restrict__ cell_cost,
                                                     __nv_bfloat16* __restrict__ out,
                                                     uint32_t* __restrict__ dims) {
  __shared__ uint32_t blocked_sum[kCells], all_sum[kCells];
  const uint32_t n = blockIdx.x;
  if (n >= count) return;
  const int tid = threadIdx.x;
  const apgar_b200_lattice_net net = nets[n];
  const int w = static_cast<int>(net.win_w), h = static_cast<int>(net.win_h);
  int s = 2;
  while ((((w > h ? w : h) - 1) >> s) >= kGrid - 1) ++s;  // at most 63 coarse cells a side
  const int cw = (w + (1 << s) - 1) >> s, ch = (h + (1 << s) - 1) >> s;
  if (tid == 0) dims[n] = static_cast<uint32_t>(cw) | (static_cast<uint32_t>(ch) << 8) |
                          (static_cast<uint32_t>(s) << 16);
  const int rows = min(ch, kGrid - 1) + 1;  // grid rows written: 0 .. ch
  for (int c = tid; c < rows * kGrid; c += blockDim.x) {
    blocked_sum[c] = 0u;
    all_sum[c] = 0u;
  }
  __syncthreads();
  const int x0w = static_cast<int>(net.win_x0), y0w = static_cast<int>(net.win_y0);
  const int wlo = x0w >> 5, nw = ((x0w + w - 1) >> 5) - wlo + 1;
  for (int u = tid; u < h * nw; u += blockDim.x) {
    const int y = u / nw, wi = wlo + u % nw;
    // window columns of this word, and the coarse cells they fall in
    const int fx0 = max(0, (wi << 5) - x0w), fx1 = min(w, (wi << 5) + 32 - x0w);
    const int cx0 = fx0 >> s, cx1 = (fx1 - 1) >> s;  // at most 9 coarse cells (s >= 2)
    uint32_t m[9], b[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const int cx = cx0 + j;
      const int lo = max(fx0, cx << s) + x0w - (wi << 5), hi = min(fx1, (cx + 1) << s) + x0w - (wi << 5);
      m[j] = cx <= cx1 ? (hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u)) & ~((1u << lo) - 1u) : 0u;
      b[j] = 0u;
    }
    const uint32_t* word = lat.blocked + static_cast<size_t>(y0w + y) * lat.words + wi;
    const size_t layer_stride = static_cast<size_t>(lat.height) * lat.words;
    uint32_t all = 0xFFFFFFFFu;
#pragma unroll 4
    for (int l = 0; l < lat.layers; ++l) {
      const uint32_t v = __ldg(word + l * layer_stride);
      all &= v;
#pragma unroll
      for (int j = 0; j < 9; ++j) b[j] += __popc(v & m[j]);
    }
    const int cy = y >> s;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      // m[j] is zero past cx1: nothing is added there
      if (b[j] != 0u) atomicAdd(&blocked_sum[cy * kGrid + cx0 + j], b[j]);
      const uint32_t a = __popc(all & m[j]);
      if (a != 0u) atomicAdd(&all_sum[cy * kGrid + cx0 + j], a);
    }
  }
  __syncthreads();
  const float scx = static_cast<float>((static_cast<int>(net.start_x) - x0w) >> s);
  const float scy = static_cast<float>((static_cast<int>(net.start_y) - y0w) >> s);
  const float gcx = static_cast<float>((static_cast<int>(net.goal_x) - x0w) >> s);
  const float gcy = static_cast<float>((static_cast<int>(net.goal_y) - y0w) >> s);
  const float sgx = gcx - scx, sgy = gcy - scy;
  const float seg2 = sgx * sgx + sgy * sgy;
  for (int c = tid; c < (rows + 1) * kGrid; c += blockDim.x) {
    const int cy = c / kGrid - 1, cx = c % kGrid;  // row -1: the zero pad row above the grid
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = 0.f;
    if (cx < cw && cy >= 0 && cy < ch) {
      const int x0 = cx << s, x1 = min(w, (cx + 1) << s);
      const int y0 = cy << s, y1 = min(h, (cy + 1) << s);
      const float cells = static_cast<float>((x1 - x0) * (y1 - y0));
      v[0] = static_cast<float>(blocked_sum[cy * kGrid + cx]) / (cells * static_cast<float>(lat.layers));
      v[1] = static_cast<float>(all_sum[cy * kGrid + cx]) / cells;
      if (cell_cost != nullptr) {
        // congestion: mean entry price over a sample of at most 4 x 4 cells per layer
        const int step = max(1, (1 << s) / 4);
        float sum = 0.f, k = 0.f;
        for (int l = 0; l < lat.layers; ++l) {
          for (int y = y0; y < y1; y += step) {
            for (int x = x0; x < x1; x += step) {
              const size_t gi = (static_cast<size_t>(l) * lat.height + (net.win_y0 + y)) * lat.width +
                                (net.win_x0 + x);
              sum += fminf(static_cast<float>(__ldg(cell_cost + gi)), 65535.f);
              k += 1.f;
            }
          }
        }
        v[2] = fminf(sum / (k * 1024.f), 8.f);
      }
      const float fx = static_cast<float>(cx), fy = static_cast<float>(cy);
      v[3] = (fx == scx && fy == scy) ? 1.f : 0.f;
      v[4] = (fx == gcx && fy == gcy) ? 1.f : 0.f;
      v[5] = 1.f;
      v[6] = (fx - scx) / 32.f;
      v[7] = (fy - scy) / 32.f;
      v[8] = (fx - gcx) / 32.f;
      v[9] = (fy - gcy) / 32.f;
      // distance to the start-goal segment, in coarse cells
      float t = seg2 > 0.f ? ((fx - scx) * sgx + (fy - scy) * sgy) / seg2 : 0.f;
      t = fminf(fmaxf(t, 0.f), 1.f);
      const float ex = fx - (scx + t * sgx), ey = fy - (scy + t * sgy);
      v[10] = fminf(sqrtf(ex * ex + ey * ey) / 8.f, 4.f);
    }
    uint4* dst = reinterpret_cast<uint4*>(out + act_cell(n, cy, cx) * kCin0);
    dst[0] = pack8(v);
    dst[1] = pack8(v + 8);
  }
}

// Coarse training labels: 1 where the net's reached path has a cell.
__global__ void labels_kernel(const apgar_b200_lattice_net* __restrict__ nets, uint32_t count,
                              const uint32_t* __restrict__ dims, int lat_w, int lat_h,
                              const apgar_b200_lattice_result* __restrict__ results,
                              const uint32_t* __restrict__ paths, uint8_t* __restrict__ labels) {
  const uint32_t n = blockIdx.x;
  if (n >= count) return;
  uint8_t* lab = labels + static_cast<size_t>(n) * kCells;
  for (int c = threadIdx.x; c < kCells; c += blockDim.x) lab[c] = 0;
  __syncthreads();
  const apgar_b200_lattice_result r = results[n];
  if (r.completion != APGAR_B200_COMPLETION_REACHED) return;
  const int s = static_cast<int>(dims[n] >> 16);
  const apgar_b200_lattice_net net = nets[n];
  for (uint32_t j = threadIdx.x; j < r.path_len; j += blockDim.x) {
    const uint32_t c = paths[r.path_offset + j];
    const int x = static_cast<int>(c % static_cast<uint32_t>(lat_w)) - static_cast<int>(net.win_x0);
    const int y = static_cast<int>((c / static_cast<uint32_t>(lat_w)) % static_cast<uint32_t>(lat_h)) -
                  static_cast<int>(net.win_y0);
    if (x >= 0 && y >= 0 && x < static_cast<int>(net.win_w) && y < static_cast<int>(net.win_h)) {
      lab[(y >> s) * kGrid + (x >> s)] = 1;
    }
  }
}

// ------------------------ 3x3 conv on tensor cores -------------------------

struct ConvArgs {
  const __nv_bfloat16* x;     // [n][64][64][cin]
  const __nv_bfloat16* w;     // [32][9 * cin], k = tap * cin + ci, tap = (dy + 1) * 3 + dx + 1
  const float* bias;          // kRelu: [32]
  const __nv_bfloat16* gate;  // kGate: [n][64][64][32]; output *= (gate > 0)
  __nv_bfloat16* y;           // [n][64][64][32]
  const uint32_t* dims;
  uint32_t count;
  uint32_t* error;
};

enum { kEpiRelu = 0, kEpiGate = 1 };

// The input halo of a 128-cell tile (rows y0 - 1 .. y0 + 2, columns -1 .. 64
// of one net): [4][66][cin] bf16, zero outside the window.
template <int CIN>
struct Halo {
  static constexpr int kCols = kGrid + 2;
  static constexpr int kUnits = 4 * kCols * (CIN / 8);  // 16-byte chunks
  static constexpr int kBytes = kUnits * 16;
};

// Stages a tile's halo with every load of a thread in flight before its
// first store (one exposed latency per tile instead of one per chunk).
template <int CIN>
__device__ __forceinline__ void stage_halo(const __nv_bfloat16* x, uint32_t net, int y0, int cw, int ch,
                                           uint8_t* halo, int tid) {
  constexpr int kUnits = Halo<CIN>::kUnits;
  constexpr int kPer = (kUnits + 127) / 128;
  uint4 v[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int u = tid + k * 128;
    v[k] = make_uint4(0u, 0u, 0u, 0u);
    if (u < kUnits) {
      const int j = u % (CIN / 8), rest = u / (CIN / 8);
      const int c = rest % Halo<CIN>::kCols, r = rest / Halo<CIN>::kCols;
      const int sy = y0 - 1 + r, sx = c - 1;
      if (sx >= 0 && sy >= 0 && sx < cw && sy < ch) {
        v[k] = __ldg(reinterpret_cast<const uint4*>(x + act_cell(net, sy, sx) * CIN) + j);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int u = tid + k * 128;
    if (u < kUnits) reinterpret_cast<uint4*>(halo)[u] = v[k];
  }
}

// Halo chunk j of the input cell read by output cell m (0..127) through tap t.
template <int CIN>
__device__ __forceinline__ uint4 halo_chunk(const uint8_t* halo, int m, int t, int j) {
  const int r = m / kGrid + t / 3, c = m % kGrid + t % 3;
  return reinterpret_cast<const uint4*>(halo)[(r * Halo<CIN>::kCols + c) * (CIN / 8) + j];
}

// The forward conv's operands.  A: the tile's four input rows (y0 - 1 ..
// y0 + 2, 64 cells each) staged as CIN / 8 planes of 16-byte chunks (8
// channels of one cell).  Each plane is [128-byte lead][256 cells][128-byte
// tail]; the last chunk of the lead and the first of the tail are zero guard
// cells.  The A operand of tap (dy, dx) for the 128 output cells is the
// staged run that starts at cell (1 + dy) * 64 + dx: K-major, 8-cell groups
// 128 bytes apart (SBO), the two chunks of a K = 16 step one plane apart
// (LBO).  No im2col copy.  B: the weights, [32 rows][9 * CIN], K-major.  A
// narrow tile (a window at most 31 columns wide) stages rows y0 - 1 .. y0 + 4
// of 32 cells instead and its runs use a 32-cell row pitch.
//
// Roles (warp-specialised, 192 threads): warp 4 lane 0 loads stages with TMA
// (a 3-D tensor map over the NHWC tensor, {8 channels, chunk, cell}, whose
// box {8, 1, 256} lands one plane: the NHWC -> planar transposition is done
// by the copy engine; narrow tiles through a 4-D map, box {8, 1, 32, 6});
// warp 5 lane 0 issues the MMAs; warps 0-3 (TMEM lanes 0-127) drain the
// accumulators and store each warp's 32 cells through a 512-byte shared slot
// (every store instruction 512 contiguous bytes).  Stages and accumulators
// form rings handed over by mbarriers, so loads, MMAs and epilogues of
// different tiles overlap.
// Pipeline depth: stages (A tiles in flight) and accumulators per CTA, CTAs
// per SM.
constexpr int kConvStages = 3, kConvAccs = 2, kConvPerSm = 3;
static_assert((kConvAccs & (kConvAccs - 1)) == 0, "TMEM allocations are powers of two columns");

template <int CIN>
struct ConvSmem {
  static constexpr int K = 9 * CIN;
  static constexpr int kChunks = K / 8;                 // 16-byte chunks per B row
  static constexpr int kSboB = kChunks * 128;           // bytes between 8-row groups of B
  static constexpr int kBytesB = 4 * kSboB;             // 32 rows
  static constexpr int kLead = 128;                     // plane bytes before cell 0
  static constexpr int kPlane = kLead + 4 * kGrid * 16 + 128;
  static constexpr int kBytesA = (CIN / 8) * kPlane;
  static constexpr int kTx = (CIN / 8) * 4 * kGrid * 16;  // TMA bytes per stage, 64-cell rows
  static constexpr int kTxNarrow = (CIN / 8) * 6 * (kGrid / 2) * 16;  // 32-cell rows
  static constexpr int kStages = kConvStages;
  static constexpr int kAccs = kConvAccs;               // 32-column accumulators
  static constexpr int kOffB = kStages * kBytesA;
  static constexpr int kOffBias = kOffB + kBytesB;      // 32 f32
  static constexpr int kOffOut = kOffBias + 128;        // [4 warps][512 B] store staging
  static constexpr int kOffBar = kOffOut + 4 * 512;     // full, empty, accfull, accempty
  static constexpr int kBytes = kOffBar + 8 * (2 * kStages + 2 * kAccs);
  static_assert(kPlane % 128 == 0 && kBytesA % 128 == 0, "TMA destinations are 128-byte aligned");
};

constexpr int kConvThreads = 192;
constexpr int kEpiWarps = 4;

__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// One plane of a stage: box {8, 1, 256} at {0, chunk, cell} of the tensor map.
__device__ __forceinline__ void tma_load_plane(uint32_t dst, const CUtensorMap* map, int chunk, int cell,
                                               uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(chunk), "r"(cell), "r"(bar)
      : "memory");
}

// Rows y0 - 1 .. y0 + 4, columns 0 .. 31 of one chunk: box {8, 1, 32, 6} at
// {0, chunk, 0, padded row} of the narrow tensor map.
__device__ __forceinline__ void tma_load_plane_narrow(uint32_t dst, const CUtensorMap* map, int chunk, int row,
                                                      uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(chunk), "r"(0), "r"(row), "r"(bar)
      : "memory");
}

// Tile `item` of the conv (net = item / 32, j = item % 32).  A net whose
// window is at most 31 coarse columns wide takes tiles of four 32-cell rows
// (y0 = 4j, j < 16): its column 31 is outside the window and zero, so the
// shifted-run operands work with a 32-cell pitch, and the MMA work on columns
// 32 .. 63 is skipped.  A wider net takes tiles of two 64-cell rows
// (y0 = 2j).  A tile exists when y0 <= ch.
struct ConvTile {
  uint32_t net;
  int y0;
  int pitch;  // cells per tile row: 32 or 64
};
__device__ __forceinline__ bool conv_tile(const uint32_t* dims, uint32_t item, ConvTile& t) {
  t.net = item / (kGrid / 2);
  const int j = static_cast<int>(item % (kGrid / 2));
  const uint32_t d = __ldg(dims + t.net);
  const bool narrow = static_cast<int>(dims_w(d)) < kGrid / 2;
  t.pitch = narrow ? kGrid / 2 : kGrid;
  t.y0 = narrow ? 4 * j : 2 * j;
  return (!narrow || j < kGrid / 4) && t.y0 <= static_cast<int>(dims_h(d));
}

// The next tile of this CTA's strided item sequence from `item` on, or
// `items` when there is none.
__device__ __forceinline__ uint32_t next_conv_item(const uint32_t* dims, uint32_t item, uint32_t items) {
  ConvTile t;
  for (; item < items; item += gridDim.x) {
    if (conv_tile(dims, item, t)) return item;
  }
  return items;
}

// out[cell][co] = epilogue(sum_{tap, ci} x[cell + tap][ci] * w[co][tap][ci]).
// `xmap`: the input as {8 channels, CIN / 8 chunks, count * 66 * 64 cells};
// `nmap`: the same as {8 channels, CIN / 8 chunks, 64 columns, count * 66 rows}.
template <int CIN, int EPI>
__global__ void __launch_bounds__(kConvThreads) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                                  const __grid_constant__ CUtensorMap nmap,
                                                                  ConvArgs a) {
  using S = ConvSmem<CIN>;
  constexpr int kSt = S::kStages, kAc = S::kAccs;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sb = smem + S::kOffB;
  float* sbias = reinterpret_cast<float*>(smem + S::kOffBias);
  const uint32_t bar0 = smem_addr(smem + S::kOffBar);
  // barrier addresses: full[s], empty[s], accfull[q], accempty[q]
  const auto full = [&](int st) { return bar0 + 8u * static_cast<uint32_t>(st); };
  const auto empty = [&](int st) { return bar0 + 8u * static_cast<uint32_t>(kSt + st); };
  const auto accfull = [&](int q) { return bar0 + 8u * static_cast<uint32_t>(2 * kSt + q); };
  const auto accempty = [&](int q) { return bar0 + 8u * static_cast<uint32_t>(2 * kSt + kAc + q); };
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ uint32_t loaded, waited;  // stages loaded / whose loads the MMA role waited for
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // weights: the resident B operand (N = 32 rows, K-major)
  for (int u = tid; u < 32 * S::kChunks; u += kConvThreads) {
    const int n = u / S::kChunks, c = u % S::kChunks;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.w + static_cast<size_t>(n) * S::K) + c);
    *reinterpret_cast<uint4*>(sb + (n % 8) * 16 + (n / 8) * S::kSboB + c * 128) = v;
  }
  if constexpr (EPI == kEpiRelu) {
    if (tid < 32) sbias[tid] = __ldg(a.bias + tid);
  }
  // the guard cells of every plane of every stage stay zero (TMA writes cells only)
  for (int u = tid; u < 2 * kSt * (CIN / 8); u += kConvThreads) {
    const int plane = u >> 1;  // stage * (CIN / 8) + chunk
    *reinterpret_cast<uint4*>(smem + plane * S::kPlane +
                              ((u & 1) ? S::kLead + 4 * kGrid * 16 : S::kLead - 16)) =
        make_uint4(0u, 0u, 0u, 0u);
  }
  if (warp == 5) tmem_alloc(&tmem_slot, 32 * kAc);
  if (tid == 0) {
    for (int st = 0; st < kSt; ++st) {
      bar_init(full(st), 1);
      bar_init(empty(st), 1);
    }
    for (int q = 0; q < kAc; ++q) {
      bar_init(accfull(q), 1);
      bar_init(accempty(q), 32 * kEpiWarps);
    }
    abort_flag = 0;
    loaded = waited = 0;
  }
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t items = a.count * (kGrid / 2);
  const volatile int* abort_v = &abort_flag;
  // a bounded wait; on expiry every role stops at its next check
  const auto wait = [&](uint32_t bar, uint32_t parity) {
    if (bar_wait(bar, parity)) return true;
    atomicExch(&abort_flag, 1);
    return false;
  };

  if (warp == 4) {
    // ---- producer: one thread, four (two) plane loads per stage ----
    if (lane == 0) {
      uint32_t k = 0;
      for (uint32_t item = next_conv_item(a.dims, blockIdx.x, items); item < items;
           item = next_conv_item(a.dims, item + gridDim.x, items), ++k) {
        const int st = static_cast<int>(k % kSt);
        if (*abort_v || !wait(empty(st), ((k / kSt) & 1u) ^ 1u)) break;
        ConvTile tile;
        conv_tile(a.dims, item, tile);
        const int row = static_cast<int>(tile.net * kPadRows + tile.y0);  // padded index of row y0 - 1
        const uint32_t dst = smem_addr(smem + st * S::kBytesA) + S::kLead;
        if (tile.pitch == kGrid) {
          bar_expect_tx(full(st), S::kTx);
#pragma unroll
          for (int j = 0; j < CIN / 8; ++j) tma_load_plane(dst + j * S::kPlane, &xmap, j, row * kGrid, full(st));
        } else {
          bar_expect_tx(full(st), S::kTxNarrow);
#pragma unroll
          for (int j = 0; j < CIN / 8; ++j) tma_load_plane_narrow(dst + j * S::kPlane, &nmap, j, row, full(st));
        }
      }
      loaded = k;
    }
  } else if (warp == 5) {
    // ---- MMA issuer: one thread, 9 taps x CIN / 16 K-steps per tile ----
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(128, 32, 0, 0);
      const uint32_t b0 = smem_addr(sb);
      uint32_t k = 0, consumed = 0;
      for (uint32_t item = next_conv_item(a.dims, blockIdx.x, items); item < items;
           item = next_conv_item(a.dims, item + gridDim.x, items), ++k) {
        const int st = static_cast<int>(k % kSt), q = static_cast<int>(k % kAc);
        if (*abort_v || !wait(full(st), (k / kSt) & 1u)) break;
        ++consumed;
        if (!wait(accempty(q), ((k / kAc) & 1u) ^ 1u)) break;
        fence_after_sync();
        ConvTile tile;
        conv_tile(a.dims, item, tile);
        const uint32_t a0 = smem_addr(smem + st * S::kBytesA) + S::kLead;
        const uint32_t acc = tmem + static_cast<uint32_t>(q * 32);
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          const int off = (t / 3) * tile.pitch + (t % 3 - 1);  // staged cell of output 0
#pragma unroll
          for (int jj = 0; jj < CIN / 16; ++jj) {
            const int kk = t * (CIN / 16) + jj;
            mma_bf16(acc, umma_desc(a0 + 2 * jj * S::kPlane + off * 16, S::kPlane, 128),
                     umma_desc(b0 + kk * 256, 128, S::kSboB), idesc, kk > 0 ? 1u : 0u);
          }
        }
        mma_commit(empty(st));  // the stage is free once these MMAs have read it
        mma_commit(accfull(q));
      }
      waited = consumed;
      // the last tile's MMAs (all earlier ones complete before it) are done
      // before the CTA can free its tensor memory
      if (k > 0) wait(accfull(static_cast<int>((k - 1) % kAc)), ((k - 1) / kAc) & 1u);
    }
  } else {
    // ---- epilogue: warps 0-3, thread = accumulator row = cell m ----
    uint32_t k = 0;
    for (uint32_t item = next_conv_item(a.dims, blockIdx.x, items); item < items;
         item = next_conv_item(a.dims, item + gridDim.x, items), ++k) {
      const int q = static_cast<int>(k % kAc);
      const bool ok = !*abort_v && wait(accfull(q), (k / kAc) & 1u);
      if (__any_sync(0xFFFFFFFFu, !ok)) break;  // warp-uniform: tcgen05.ld is .sync.aligned
      fence_after_sync();
      float o[32];
      tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(q * 32), o);
      fence_before_sync();
      bar_arrive(accempty(q));
      ConvTile tile;
      conv_tile(a.dims, item, tile);
      const uint32_t net = tile.net;
      const int y0 = tile.y0;
      const uint32_t d = __ldg(a.dims + net);
      const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
      const int m = warp * 32 + lane;
      const int py = y0 + m / tile.pitch, px = m % tile.pitch;
      const size_t cell = act_cell(net, py, px);
      // cells outside the window are written as zeros (the layout's invariant)
      if (px < cw && py < ch) {
        if constexpr (EPI == kEpiRelu) {
#pragma unroll
          for (int c4 = 0; c4 < 8; ++c4) {
            const float4 b4 = reinterpret_cast<const float4*>(sbias)[c4];
            o[4 * c4 + 0] = fmaxf(o[4 * c4 + 0] + b4.x, 0.f);
            o[4 * c4 + 1] = fmaxf(o[4 * c4 + 1] + b4.y, 0.f);
            o[4 * c4 + 2] = fmaxf(o[4 * c4 + 2] + b4.z, 0.f);
            o[4 * c4 + 3] = fmaxf(o[4 * c4 + 3] + b4.w, 0.f);
          }
        } else {
          const uint4* g = reinterpret_cast<const uint4*>(a.gate + cell * kCh);
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            float gv[8];
            unpack8(__ldg(g + qq), gv);
#pragma unroll
            for (int i = 0; i < 8; ++i) o[qq * 8 + i] = gv[i] > 0.f ? o[qq * 8 + i] : 0.f;
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) o[c] = 0.f;
      }
      // A warp's 32 cells are 32 consecutive cells of one row (2 KB).  They
      // go out through a 512-byte staging slot, eight cells per pass, so that
      // every store instruction writes 512 contiguous bytes.
      uint4 pk[4];
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) pk[qq] = pack8(o + qq * 8);
      const int m0 = warp * 32;
      const int py0 = y0 + m0 / tile.pitch, px0 = m0 % tile.pitch;
      uint4* slot = reinterpret_cast<uint4*>(smem + S::kOffOut + warp * 512);
      uint4* dst = reinterpret_cast<uint4*>(a.y + act_cell(net, py0, px0) * kCh);
      const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
      for (int pass = 0; pass < 4; ++pass) {
        if ((lane >> 3) == pass) {
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) slot[(lane & 7) * 4 + qq] = pk[qq];
        }
        __syncwarp();
        dst[pass * 32 + lane] = slot[lane];
        __syncwarp();
      }
      // (a narrow tile's columns 32 .. 63 are left as they are: only narrow
      // tiles, which never read them, consume this net's activations)
      if (y0 == 0 && m0 < tile.pitch) {
        // the zero pad row above the grid
        uint4* pad = reinterpret_cast<uint4*>(a.y + act_cell(net, -1, px0) * kCh);
#pragma unroll
        for (int pass = 0; pass < 4; ++pass) pad[pass * 32 + lane] = zero;
      }
    }
  }
  __syncthreads();
  if (warp == 4 && lane == 0) {
    // loads nobody waited for (only after an expired wait): let them land
    // before the CTA's shared memory goes away
    for (uint32_t k = waited; k < loaded; ++k) {
      bar_wait(full(static_cast<int>(k % kSt)), (k / kSt) & 1u);
    }
  }
  if (tid == 0 && abort_flag) atomicOr(a.error, APGAR_B200_CNN_TIMEOUT);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 5) tmem_free(tmem, 32 * kAc);
}

// ------------------- weight gradient on tensor cores ----------------------

struct WgradArgs {
  const __nv_bfloat16* x;   // layer input [n][64][64][cin]
  const __nv_bfloat16* dy;  // gradient at the layer's pre-activation [n][64][64][32]
  const uint32_t* dims;
  uint32_t count;
  float* dw;                // [32][9 * cin] (added to)
  float* db;                // [32] (added to)
  uint32_t* error;
};

template <int CIN>
struct WgradSmem {
  static constexpr int K = 9 * CIN;                    // rows of D
  static constexpr int kTiles = (K + 127) / 128;       // M tiles of 128 rows
  static constexpr int kSbo = 2048;                    // 16 K-groups x 128 bytes
  static constexpr int kBytesTile = 16 * kSbo;         // 128 rows x 128 cells
  static constexpr int kBytesA = kTiles * kBytesTile;
  static constexpr int kBytesB = 4 * kSbo;             // 32 rows x 128 cells
  static constexpr int kBytes = kBytesA + kBytesB + Halo<CIN>::kBytes + 16;
};

// dw[co][tap * CIN + ci] += sum over cells of x[cell + tap][ci] * dy[cell][co];
// db[co] += sum over cells of dy[cell][co].  Operands MN-major: element
// (row r, cell k) at (r % 8) * 2 + (k % 8) * 16 + (r / 8) * SBO + (k / 8) * 128.
template <int CIN>
__global__ void __launch_bounds__(128) conv_wgrad_tc_kernel(WgradArgs a) {
  using S = WgradSmem<CIN>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sa = smem;
  uint8_t* sb = smem + S::kBytesA;
  uint8_t* halo = smem + S::kBytesA + S::kBytesB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S::kBytesA + S::kBytesB + Halo<CIN>::kBytes);
  __shared__ uint32_t tmem_slot;
  __shared__ float bias_part[32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // rows K .. kTiles * 128 of the last tile stay zero
  for (int u = tid; u < S::kBytesA / 16; u += 128) reinterpret_cast<uint4*>(sa)[u] = make_uint4(0, 0, 0, 0);
  if (tid < 32) bias_part[tid] = 0.f;
  if (warp == 0) tmem_alloc(&tmem_slot, 128);
  if (tid == 0) bar_init(smem_addr(bar), 1);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = idesc_bf16(128, 32, 1, 1);
  uint32_t phase = 0;
  bool failed = false, any = false;
  float bsum = 0.f;  // this thread's share of db (co = tid % 32)

  const uint32_t items = a.count * (kGrid / 2);
  for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
    const uint32_t net = item / (kGrid / 2);
    const int y0 = static_cast<int>(item % (kGrid / 2)) * 2;
    const uint32_t d = a.dims[net];
    const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
    if (y0 >= ch) continue;
    // B: dy chunks (8 channels) per cell; zero outside the window
    for (int u = tid; u < 128 * 4; u += 128) {
      const int k = u % 128, j = u / 128;
      const int py = y0 + k / kGrid, px = k % kGrid;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (px < cw && py < ch) v = __ldg(reinterpret_cast<const uint4*>(a.dy + act_cell(net, py, px) * kCh) + j);
      *reinterpret_cast<uint4*>(sb + (k % 8) * 16 + j * S::kSbo + (k / 8) * 128) = v;
    }
    // A: im2col rows (tap, ci) per cell, from the staged halo (cells outside
    // the window carry finite halo values against a zero dy)
    stage_halo<CIN>(a.x, net, y0, cw, ch, halo, tid);
    __syncthreads();
    for (int u = tid; u < 128 * 9 * (CIN / 8); u += 128) {
      const int k = u % 128, r = u / 128;
      const int j = r % (CIN / 8), t = r / (CIN / 8);
      const uint4 v = halo_chunk<CIN>(halo, k, t, j);
      const int row = t * CIN + j * 8;
      *reinterpret_cast<uint4*>(sa + (row / 128) * S::kBytesTile + (k % 8) * 16 + ((row % 128) / 8) * S::kSbo +
                                (k / 8) * 128) = v;
    }
    fence_async_smem();
    __syncthreads();
    // bias gradient from the staged dy (thread: channel tid % 32, cells tid / 32 + 4 i)
    {
      const int c = tid % 32;
      for (int k = tid / 32; k < 128; k += 4) {
        const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(
            sb + (k % 8) * 16 + (c / 8) * S::kSbo + (k / 8) * 128) + (c % 8);
        bsum += __bfloat162float(*e);
      }
    }
    if (tid == 0) {
      fence_after_sync();
      const uint32_t b0 = smem_addr(sb);
#pragma unroll 1
      for (int mt = 0; mt < S::kTiles; ++mt) {
        const uint32_t a0 = smem_addr(sa) + mt * S::kBytesTile;
#pragma unroll 1
        for (int kk = 0; kk < 8; ++kk) {
          mma_bf16(tmem + mt * 32, umma_desc(a0 + kk * 256, 128, S::kSbo),
                   umma_desc(b0 + kk * 256, 128, S::kSbo), idesc, (any || kk > 0) ? 1u : 0u);
        }
      }
      mma_commit(smem_addr(bar));
    }
    any = true;
    const bool ok = bar_wait(smem_addr(bar), phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
  }
  if (failed) {
    if (tid == 0) atomicOr(a.error, APGAR_B200_CNN_TIMEOUT);
    bar_wait(smem_addr(bar), phase);
  } else if (any) {
    fence_after_sync();
    for (int mt = 0; mt < S::kTiles; ++mt) {
      float v[32];
      tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + mt * 32, v);
      const int row = mt * 128 + warp * 32 + lane;
      if (row < S::K) {
#pragma unroll
        for (int c = 0; c < 32; ++c) atomicAdd(a.dw + c * S::K + row, v[c]);
      }
    }
    atomicAdd(&bias_part[tid % 32], bsum);
  }
  fence_before_sync();
  __syncthreads();
  if (!failed && any && tid < 32) atomicAdd(a.db + tid, bias_part[tid]);
  if (warp == 0) tmem_free(tmem, 128);
}

// ------------------------------ head + loss -------------------------------

// logit[cell] = b6 + sum_{tap, ci} w6[tap][ci] * act[cell + tap][ci] (FP32,
// taps outside the window skipped, outside cells 0).  A block takes one band
// of kHeadRows rows of one net: it stages the band's rows and their halo
// (rows y0 - 1 .. y0 + kHeadRows, window rows only) in shared memory with
// cp.async, the 16-byte chunks of a cell rotated by its column (chunk q of
// cell x at slot q ^ (x & 3)) so that a warp's 32 neighbouring cells read
// conflict-free; each thread then sums its cells' 288 products in the same
// order as a plain per-cell loop.
constexpr int kHeadRows = 8;
constexpr int kHeadBands = kGrid / kHeadRows;
constexpr int kHeadStageRows = kHeadRows + 2;
constexpr int kHeadSmem = kHeadStageRows * kGrid * kCh * 2;

__global__ void __launch_bounds__(256, 3) head_forward_kernel(const __nv_bfloat16* __restrict__ act,
                                                           const float* __restrict__ w6,
                                                           const float* __restrict__ b6,
                                                           const uint32_t* __restrict__ dims, uint32_t count,
                                                           float* __restrict__ logits) {
  extern __shared__ __align__(16) uint8_t hs[];  // [kHeadStageRows][64 cells][4 chunks]
  __shared__ __align__(16) float ws[9 * kCh];
  const uint32_t net = blockIdx.x / kHeadBands;
  const int y0 = static_cast<int>(blockIdx.x % kHeadBands) * kHeadRows;
  if (net >= count) return;
  const uint32_t d = dims[net];
  const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
  float* out = logits + grid_cell(net, y0, 0);
  if (y0 >= ch) {  // uniform: a band below the window
    for (int i = threadIdx.x; i < kHeadRows * kGrid; i += blockDim.x) out[i] = 0.f;
    return;
  }
  for (int i = threadIdx.x; i < 9 * kCh; i += blockDim.x) ws[i] = w6[i];
  // window rows of the halo: y0 - 1 .. y0 + kHeadRows, clipped to [0, ch);
  // the first 32 columns only when the window is no wider
  const int r0 = max(y0 - 1, 0), r1 = min(y0 + kHeadRows, ch - 1);
  const int cols = cw <= kGrid / 2 ? kGrid / 2 : kGrid;
  const uint8_t* src = reinterpret_cast<const uint8_t*>(act + act_cell(net, r0, 0) * kCh);
  const int chunks = (r1 - r0 + 1) * cols * 4;
  const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(hs));
  for (int u = threadIdx.x; u < chunks; u += blockDim.x) {
    const int q = u & 3, cc = u >> 2;
    const int row = cc / cols, col = cc % cols;           // from r0
    const int c = row * kGrid + col;                      // staged cell (rows from r0)
    const int slot = (r0 - (y0 - 1)) * kGrid + c;         // stage row 0 is y0 - 1
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(base + slot * 64 + ((q ^ (c & 3)) << 4)),
                 "l"(src + (static_cast<size_t>(c) * 4 + q) * 16)
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const float bias = b6[0];
#pragma unroll 1
  for (int i = threadIdx.x; i < kHeadRows * kGrid; i += blockDim.x) {
    const int y = y0 + i / kGrid, x = i % kGrid;
    float z = 0.f;
    if (x < cw && y < ch) {
      z = bias;
#pragma unroll 1
      for (int t = 0; t < 9; ++t) {
        const int sy = y + t / 3 - 1, sx = x + t % 3 - 1;
        if (sx < 0 || sy < 0 || sx >= cw || sy >= ch) continue;
        const uint4* cell = reinterpret_cast<const uint4*>(hs + ((sy - (y0 - 1)) * kGrid + sx) * 64);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float v[8];
          unpack8(cell[q ^ (sx & 3)], v);
#pragma unroll
          for (int k = 0; k < 8; ++k) z = fmaf(ws[t * kCh + q * 8 + k], v[k], z);
        }
      }
    }
    out[i] = z;
  }
}

// Weighted binary cross-entropy on logits, averaged over each net's window
// cells and then over nets: dlogit = weight * (sigmoid(z) - y) / (cells * count).
__global__ void loss_kernel(const float* __restrict__ logits, const uint8_t* __restrict__ labels,
                            const uint32_t* __restrict__ dims, uint32_t count, float pos_weight,
                            float* __restrict__ dlogit, float* __restrict__ loss) {
  float acc = 0.f;
  const size_t total = static_cast<size_t>(count) * kCells;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t net = static_cast<uint32_t>(i / kCells);
    const int y = static_cast<int>((i / kGrid) % kGrid), x = static_cast<int>(i % kGrid);
    const uint32_t d = dims[net];
    const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
    float g = 0.f;
    if (x < cw && y < ch) {
      const float z = logits[i];
      const float t = labels[i] ? 1.f : 0.f;
      const float wgt = labels[i] ? pos_weight : 1.f;
      const float norm = 1.f / (static_cast<float>(cw * ch) * static_cast<float>(count));
      const float sig = 1.f / (1.f + __expf(-z));
      g = wgt * (sig - t) * norm;
      acc += wgt * (fmaxf(z, 0.f) - z * t + log1pf(__expf(-fabsf(z)))) * norm;
    }
    dlogit[i] = g;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(loss, acc);
}

// Head backward, one warp per cell and one lane per channel ci:
//   dact[cell][ci] = sum_tap w6[tap][ci] * dlogit[cell - tap], gated by act > 0
//   dw6[tap][ci] += dlogit[cell] * act[cell + tap][ci];  db6 += dlogit[cell]
__global__ void head_backward_kernel(const __nv_bfloat16* __restrict__ act, const float* __restrict__ w6,
                                     const float* __restrict__ dlogit, const uint32_t* __restrict__ dims,
                                     uint32_t count, __nv_bfloat16* __restrict__ dact,
                                     float* __restrict__ dw6, float* __restrict__ db6) {
  const int lane = threadIdx.x & 31;
  float wcol[9], acc[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    wcol[t] = w6[t * kCh + lane];
    acc[t] = 0.f;
  }
  float bacc = 0.f;
  const size_t total = static_cast<size_t>(count) * kCells;
  const size_t warps = static_cast<size_t>(gridDim.x) * (blockDim.x / 32);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x / 32) + (threadIdx.x >> 5); i < total; i += warps) {
    const uint32_t net = static_cast<uint32_t>(i / kCells);
    const int y = static_cast<int>((i / kGrid) % kGrid), x = static_cast<int>(i % kGrid);
    const uint32_t d = dims[net];
    const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
    if (y == 0) dact[act_cell(net, -1, x) * kCh + lane] = __float2bfloat16_rn(0.f);  // pad row
    if (x >= cw || y >= ch) {
      // the padded layout's zeros, through row ch (read by the next conv's taps)
      if (y <= ch) dact[act_cell(net, y, x) * kCh + lane] = __float2bfloat16_rn(0.f);
      continue;
    }
    const float dl = dlogit[i];
    float da = 0.f;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int dy = t / 3 - 1, dx = t % 3 - 1;
      // output cell (y - dy, x - dx) reads this cell through tap t
      const int oy = y - dy, ox = x - dx;
      if (ox >= 0 && oy >= 0 && ox < cw && oy < ch) da = fmaf(wcol[t], dlogit[grid_cell(net, oy, ox)], da);
      const int sy = y + dy, sx = x + dx;
      if (sx >= 0 && sy >= 0 && sx < cw && sy < ch) {
        acc[t] = fmaf(dl, __bfloat162float(act[act_cell(net, sy, sx) * kCh + lane]), acc[t]);
      }
    }
    const float a = __bfloat162float(act[act_cell(net, y, x) * kCh + lane]);
    dact[act_cell(net, y, x) * kCh + lane] = __float2bfloat16_rn(a > 0.f ? da : 0.f);
    bacc += dl;
  }
#pragma unroll
  for (int t = 0; t < 9; ++t) atomicAdd(dw6 + t * kCh + lane, acc[t]);
  if (lane == 0) atomicAdd(db6, bacc);
}

// ------------------------------ parameters --------------------------------

// FP32 parameters: layer l (cin_l = 16 for l = 0, else 32): w [32][9][cin_l]
// then b [32]; head: w6 [9][32] then b6.
struct ParamOffsets {
  uint32_t w[5], b[5], w6, b6, total;
};

__host__ __device__ constexpr ParamOffsets param_offsets() {
  ParamOffsets o{};
  uint32_t at = 0;
  for (int l = 0; l < 5; ++l) {
    const uint32_t cin = l == 0 ? kCin0 : kCh;
    o.w[l] = at;
    at += 32 * 9 * cin;
    o.b[l] = at;
    at += 32;
  }
  o.w6 = at;
  at += 9 * kCh;
  o.b6 = at;
  at += 1;
  o.total = at;
  return o;
}

// bf16 operands: forward wf[l] = [co][tap * cin + ci]; backward (l >= 1)
// wb[l] = [ci][tap' * 32 + co] with tap' = 8 - tap (flipped kernel).
struct OperandOffsets {
  uint32_t wf[5], wb[5], total;
};

__host__ __device__ constexpr OperandOffsets operand_offsets() {
  OperandOffsets o{};
  uint32_t at = 0;
  for (int l = 0; l < 5; ++l) {
    o.wf[l] = at;
    at += 32 * 9 * (l == 0 ? kCin0 : kCh);
  }
  for (int l = 0; l < 5; ++l) {
    o.wb[l] = at;
    if (l > 0) at += 32 * 9 * kCh;
  }
  o.total = at;
  return o;
}

__global__ void prepare_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ ops) {
  constexpr ParamOffsets P = param_offsets();
  constexpr OperandOffsets O = operand_offsets();
  for (int l = 0; l < 5; ++l) {
    const int cin = l == 0 ? kCin0 : kCh;
    const int n = 32 * 9 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const float v = params[P.w[l] + i];  // i = (co * 9 + tap) * cin + ci
      ops[O.wf[l] + i] = __float2bfloat16_rn(v);
      if (l > 0) {
        const int ci = i % cin, tap = (i / cin) % 9, co = i / (9 * cin);
        ops[O.wb[l] + ci * (9 * kCh) + (8 - tap) * kCh + co] = __float2bfloat16_rn(v);
      }
    }
  }
}

__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grads,
                            float* __restrict__ m, float* __restrict__ v, uint32_t n, float lr,
                            float beta1, float beta2, float eps, float c1, float c2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// -------------------------- corridors from logits -------------------------

// The corridor bitmap of each net: a coarse cell is on when it lies in the
// window and is the start, the goal or within `dilate` cells (Chebyshev) of a
// cell whose logit exceeds the threshold; row cy of the bitmap is words
// 2 * cy (columns 0-31) and 2 * cy + 1.  Rows are 64-bit masks: the hot rows
// come from warp ballots, the dilation is shifts and ORs of whole rows.  A net
// whose window holds more than max_cells cells (all layers; 0 = no limit)
// gets an empty bitmap: no corridor, its whole window is searched at once.
__global__ void __launch_bounds__(128) corridor_kernel(const float* __restrict__ logits,
                                                       const uint32_t* __restrict__ dims,
                                                       const apgar_b200_lattice_net* __restrict__ nets,
                                                       uint32_t count, float threshold, int dilate,
                                                       uint64_t max_cells, int layers,
                                                       uint32_t* __restrict__ bits) {
  __shared__ uint64_t hot[kGrid], wide[kGrid];
  const uint32_t n = blockIdx.x;
  if (n >= count) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t* out = bits + static_cast<size_t>(n) * 128;
  if (max_cells != 0 &&
      static_cast<uint64_t>(layers) * nets[n].win_w * nets[n].win_h > max_cells) {
    out[tid] = 0u;  // 128 threads, 128 words
    return;         // uniform: the whole block
  }
  const uint32_t d = dims[n];
  const int cw = static_cast<int>(dims_w(d)), ch = static_cast<int>(dims_h(d));
  const int s = static_cast<int>(d >> 16);
  const float* z = logits + static_cast<size_t>(n) * kCells;
  for (int y = warp; y < kGrid; y += 4) {
    const bool lo = y < ch && lane < cw && z[y * kGrid + lane] > threshold;
    const bool hi = y < ch && lane + 32 < cw && z[y * kGrid + 32 + lane] > threshold;
    const uint32_t blo = __ballot_sync(0xFFFFFFFFu, lo), bhi = __ballot_sync(0xFFFFFFFFu, hi);
    if (lane == 0) hot[y] = static_cast<uint64_t>(blo) | (static_cast<uint64_t>(bhi) << 32);
  }
  __syncthreads();
  const int dl = min(dilate, kGrid - 1);  // beyond 63 every column is covered already
  if (tid < kGrid) {
    const uint64_t v = hot[tid];
    uint64_t h = 0;
    for (int dx = -dl; dx <= dl; ++dx) h |= dx >= 0 ? v >> dx : v << -dx;  // none when dilate < 0
    wide[tid] = h;
  }
  __syncthreads();
  if (tid < kGrid) {
    const int y = tid;
    uint64_t o = 0;
    for (int dy = -dl; dy <= dl; ++dy) {
      const int yy = y + dy;
      if (yy >= 0 && yy < kGrid) o |= wide[yy];  // hot rows ch .. 63 are zero
    }
    const apgar_b200_lattice_net net = nets[n];
    const int sx = (static_cast<int>(net.start_x) - static_cast<int>(net.win_x0)) >> s;
    const int sy = (static_cast<int>(net.start_y) - static_cast<int>(net.win_y0)) >> s;
    const int gx = (static_cast<int>(net.goal_x) - static_cast<int>(net.win_x0)) >> s;
    const int gy = (static_cast<int>(net.goal_y) - static_cast<int>(net.win_y0)) >> s;
    if (y == sy && sx >= 0 && sx < kGrid) o |= 1ull << sx;
    if (y == gy && gx >= 0 && gx < kGrid) o |= 1ull << gx;
    o &= y < ch ? (cw >= kGrid ? ~0ull : (1ull << cw) - 1ull) : 0ull;
    out[2 * y] = static_cast<uint32_t>(o);
    out[2 * y + 1] = static_cast<uint32_t>(o >> 32);
  }
}

// The driver's tensor-map encoder, resolved once through the runtime (no
// link against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      f = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// The conv input [count][66][64][CIN] bf16 as {8 channels, CIN / 8 chunks,
// cells}: a box {8, 1, 256} is one 16-byte chunk of 256 consecutive cells.
template <int CIN>
cudaError_t conv_input_map(const __nv_bfloat16* x, uint32_t count, CUtensorMap* map, CUtensorMap* narrow) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (encode == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(x) & 15u) != 0) return cudaErrorInvalidValue;
  const cuuint32_t elem[4] = {1, 1, 1, 1};
  // wide tiles: four 64-cell rows as 256 consecutive cells
  const cuuint64_t dims[3] = {8, CIN / 8, static_cast<cuuint64_t>(count) * kPadRows * kGrid};
  const cuuint64_t strides[2] = {16, CIN * 2};  // bytes, dims 1 and 2
  const cuuint32_t box[3] = {8, 1, 4 * kGrid};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(x), dims, strides,
                      box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  // narrow tiles: six rows of the first 32 cells
  const cuuint64_t ndims[4] = {8, CIN / 8, kGrid, static_cast<cuuint64_t>(count) * kPadRows};
  const cuuint64_t nstrides[3] = {16, CIN * 2, static_cast<cuuint64_t>(kGrid) * CIN * 2};
  const cuuint32_t nbox[4] = {8, 1, kGrid / 2, 6};
  r = encode(narrow, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(x), ndims, nstrides, nbox,
             elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, int EPI>
cudaError_t launch_conv(const ConvArgs& a, int sm_count, cudaStream_t stream) {
  using S = ConvSmem<CIN>;
  const uint32_t items = a.count * (kGrid / 2);
  if (items == 0) return cudaSuccess;
  // planes are addressed by 32-bit cell coordinates
  if (static_cast<uint64_t>(a.count) * kPadRows * kGrid > 0x7FFFFFFFull) return cudaErrorInvalidValue;
  CUtensorMap map, narrow;
  cudaError_t e = conv_input_map<CIN>(a.x, a.count, &map, &narrow);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           S::kBytes);
  if (e != cudaSuccess) return e;
  // ~71 KB of shared memory (32 channels) and 64 TMEM columns per CTA: three
  // per SM (three CTAs' pipelines per SM measured faster than two deeper ones)
  const uint32_t grid = min(items, static_cast<uint32_t>(max(sm_count, 1) * kConvPerSm));
  conv3x3_tc_kernel<CIN, EPI><<<grid, kConvThreads, S::kBytes, stream>>>(map, narrow, a);
  return cudaGetLastError();
}

template <int CIN>
cudaError_t launch_wgrad(const WgradArgs& a, int sm_count, cudaStream_t stream) {
  const int bytes = WgradSmem<CIN>::kBytes;
  cudaError_t e = cudaFuncSetAttribute(conv_wgrad_tc_kernel<CIN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  const uint32_t items = a.count * (kGrid / 2);
  const uint32_t grid = min(items, static_cast<uint32_t>(max(sm_count, 1) * 2));
  if (grid == 0) return cudaSuccess;
  conv_wgrad_tc_kernel<CIN><<<grid, 128, bytes, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

uint32_t cnn_param_count() { return param_offsets().total; }
uint32_t cnn_operand_count() { return operand_offsets().total; }

cudaError_t launch_rasters(const LatticeDeviceView& lat, const apgar_b200_lattice_net* nets,
                           uint32_t count, const uint32_t* cell_cost, void* rasters, uint32_t* dims,
                           cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  raster_kernel<<<count, 256, 0, stream>>>(lat, nets, count, cell_cost,
                                           static_cast<__nv_bfloat16*>(rasters), dims);
  return cudaGetLastError();
}

cudaError_t launch_labels(const apgar_b200_lattice_net* nets, uint32_t count, const uint32_t* dims,
                          int lat_w, int lat_h, const apgar_b200_lattice_result* results,
                          const uint32_t* paths, uint8_t* labels, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  labels_kernel<<<count, 256, 0, stream>>>(nets, count, dims, lat_w, lat_h, results, paths, labels);
  return cudaGetLastError();
}

cudaError_t launch_prepare(const float* params, void* operands, cudaStream_t stream) {
  prepare_kernel<<<64, 256, 0, stream>>>(params, static_cast<__nv_bfloat16*>(operands));
  return cudaGetLastError();
}

// Forward: rasters -> acts[0..4] -> logits.  acts[l] may alias acts[l - 2].
cudaError_t launch_forward(const float* params, const void* operands, const void* rasters,
                           const uint32_t* dims, uint32_t count, void* const acts[5], float* logits,
                           uint32_t* error, int sm_count, cudaStream_t stream) {
  constexpr ParamOffsets P = param_offsets();
  constexpr OperandOffsets O = operand_offsets();
  if (count == 0) return cudaSuccess;
  const auto* ops = static_cast<const __nv_bfloat16*>(operands);
  for (int l = 0; l < 5; ++l) {
    ConvArgs a{};
    a.x = static_cast<const __nv_bfloat16*>(l == 0 ? rasters : acts[l - 1]);
    a.w = ops + O.wf[l];
    a.bias = params + P.b[l];
    a.y = static_cast<__nv_bfloat16*>(acts[l]);
    a.dims = dims;
    a.count = count;
    a.error = error;
    const cudaError_t e = l == 0 ? launch_conv<kCin0, kEpiRelu>(a, sm_count, stream)
                                 : launch_conv<kCh, kEpiRelu>(a, sm_count, stream);
    if (e != cudaSuccess) return e;
  }
  head_forward_kernel<<<count * kHeadBands, 256, kHeadSmem, stream>>>(
      static_cast<const __nv_bfloat16*>(acts[4]), params + P.w6, params + P.b6, dims, count, logits);
  return cudaGetLastError();
}

// Backward from the logits of a forward pass with five distinct act buffers.
// grads (FP32, same layout as params) must be zero on entry; scratch holds two
// gradient tensors of [count][64][64][32] bf16.
cudaError_t launch_backward(const float* params, const void* operands, const void* rasters,
                            const uint32_t* dims, uint32_t count, void* const acts[5],
                            const float* logits, const uint8_t* labels, float pos_weight,
                            float* dlogit, void* scratch0, void* scratch1, float* grads, float* loss,
                            uint32_t* error, int sm_count, cudaStream_t stream) {
  constexpr ParamOffsets P = param_offsets();
  constexpr OperandOffsets O = operand_offsets();
  if (count == 0) return cudaSuccess;
  const auto* ops = static_cast<const __nv_bfloat16*>(operands);
  const uint32_t blocks = min(static_cast<uint32_t>(max(sm_count, 1) * 8),
                              static_cast<uint32_t>((static_cast<size_t>(count) * kCells + 255) / 256));
  loss_kernel<<<blocks, 256, 0, stream>>>(logits, labels, dims, count, pos_weight, dlogit, loss);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  void* g[2] = {scratch0, scratch1};
  head_backward_kernel<<<blocks, 256, 0, stream>>>(static_cast<const __nv_bfloat16*>(acts[4]),
                                                   params + P.w6, dlogit, dims, count,
                                                   static_cast<__nv_bfloat16*>(g[0]), grads + P.w6,
                                                   grads + P.b6);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // g[cur] = gradient at layer l's pre-activation
  int cur = 0;
  for (int l = 4; l >= 0; --l) {
    WgradArgs wa{};
    wa.x = static_cast<const __nv_bfloat16*>(l == 0 ? rasters : acts[l - 1]);
    wa.dy = static_cast<const __nv_bfloat16*>(g[cur]);
    wa.dims = dims;
    wa.count = count;
    wa.dw = grads + P.w[l];
    wa.db = grads + P.b[l];
    wa.error = error;
    e = l == 0 ? launch_wgrad<kCin0>(wa, sm_count, stream) : launch_wgrad<kCh>(wa, sm_count, stream);
    if (e != cudaSuccess) return e;
    if (l == 0) break;
    ConvArgs a{};
    a.x = static_cast<const __nv_bfloat16*>(g[cur]);
    a.w = ops + O.wb[l];
    a.gate = static_cast<const __nv_bfloat16*>(acts[l - 1]);
    a.y = static_cast<__nv_bfloat16*>(g[cur ^ 1]);
    a.dims = dims;
    a.count = count;
    a.error = error;
    e = launch_conv<kCh, kEpiGate>(a, sm_count, stream);
    if (e != cudaSuccess) return e;
    cur ^= 1;
  }
  return cudaSuccess;
}

cudaError_t launch_adam(float* params, const float* grads, float* m, float* v, uint32_t step,
                        float lr, float beta1, float beta2, float eps, cudaStream_t stream) {
  const uint32_t n = param_offsets().total;
  const float c1 = 1.f - powf(beta1, static_cast<float>(step));
  const float c2 = 1.f - powf(beta2, static_cast<float>(step));
  adam_kernel<<<(n + 255) / 256, 256, 0, stream>>>(params, grads, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_corridors(const float* logits, const uint32_t* dims,
                             const apgar_b200_lattice_net* nets, uint32_t count, float threshold,
                             int dilate, uint64_t max_cells, int layers, uint32_t* bits,
                             cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  corridor_kernel<<<count, 128, 0, stream>>>(logits, dims, nets, count, threshold, dilate, max_cells,
                                             layers, bits);
  return cudaGetLastError();
}

}  // namespace apgar_b200
