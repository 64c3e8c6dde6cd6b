// gemm_bf16x3.cu -- S = O^T O on the 5th-generation tensor cores in split-BF16 form: the precision-split
// replacement of the FP64 dgemm of calc_phys_quantity.f90:240 (S_raw = O_store O_store^T).
//
// O (ns x nv FP64, one row per sample) is split per entry as O = H + L with H = bf16(O) and
// L = bf16(O - H), and S ~ H^T H + H^T L + L^T H (the L^T L term lies below the FP32 accumulator's
// resolution), accumulated in FP32 in tensor memory (TMEM).  The diagonal is recomputed exactly in
// FP64, so every decision the SR block takes on diag(S) (SR_pdposv.f90:18-140) is the FP64 one.
//
// One 128 x 256 tile of S per CTA (128 threads):
//   warp 0 lane 0  TMA producer: cp.async.bulk.tensor (128-byte swizzle) of the H and L tiles of both
//                  operands into a 2-stage shared-memory ring (96 KiB per stage);
//   warp 1 lane 0  issues tcgen05.mma kind::f16 (BF16 x BF16 -> FP32, 128 x 256 x 16) three times per
//                  16-sample slice, and tcgen05.commit to release each stage;
//   warps 0-3      epilogue: tcgen05.ld of their 32 TMEM lanes, FP64 stores of the strict upper triangle.
// Both operands are the same K-major arrays (H^T, L^T: [nv_pad][k_pad] BF16, samples contiguous), so a
// tile of either operand is a plain 2-D box.  No cluster multicast is used.
// Every mbarrier wait is bounded; a wait that runs out sets *err, the kernel still waits (bounded) for
// its own copies and MMAs, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

void rbmpp_note_launch();  // capi.cu: counts kernel launches

#include "tma.cuh"

namespace {

constexpr int BM = 128, BN = 256, BK = 64, ST = 2;
constexpr uint32_t A_BYTES = BM * BK * 2;                    // 16 KiB: 128 rows x 128 B
constexpr uint32_t B_BYTES = BN * BK * 2;                    // 32 KiB: 256 rows x 128 B
constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // H and L of both operands: 96 KiB
constexpr uint32_t BAR_BYTES = 128;
constexpr uint32_t SMEM_BYTES = ST * STAGE_BYTES + BAR_BYTES + 1024;  // + alignment slack
constexpr uint32_t TMEM_COLS = 256;                                   // 128 lanes x 256 FP32 columns
// instruction descriptor, kind::f16: FP32 accumulator (bit 4), A and B BF16 (bits 7, 10), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

// shared-memory matrix descriptor of a K-major tile with 128-byte swizzle: rows of 128 B, 8-row groups
// 1024 B apart (stride byte offset), leading byte offset unused (1), descriptor version 1, layout 2
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tma_load_2d(void* sdst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(sdst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  const uint32_t z = 0;  // no output lane disabled
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

// arrives once on bar when every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ bool wait_long(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < (1 << 26); it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__global__ void __launch_bounds__(128, 1)
    syrk_bf16x3_kernel(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo, int nv,
                       int kblocks, double* __restrict__ S, int* err) {
  const int i0 = blockIdx.x * BM, j0 = blockIdx.y * BN;
  if (i0 >= nv || j0 >= nv || i0 > j0 + BN - 2) return;  // no strict-upper entry in this tile
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* full = (uint64_t*)(smem + ST * STAGE_BYTES);
  uint64_t* empty = full + ST;
  uint64_t* accum = empty + ST;
  uint32_t* tmem_slot = (uint32_t*)(accum + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    int issued = 0;
    for (int kb = 0; kb < kblocks; kb++) {
      const int s = kb % ST, n = kb / ST;
      if (n > 0 && !mbar_wait(&empty[s], (uint32_t)((n - 1) & 1))) {
        *abort_flag = 1;
        break;
      }
      if (*abort_flag) break;
      uint8_t* st = smem + s * STAGE_BYTES;
      const int x = kb * BK;
      mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
      tma_load_2d(st, &tm_hi, x, i0, &full[s]);                                 // A = H rows i0..i0+127
      tma_load_2d(st + A_BYTES, &tm_lo, x, i0, &full[s]);                       // A = L
      tma_load_2d(st + 2 * A_BYTES, &tm_hi, x, j0, &full[s]);                   // B = H rows j0..j0+127
      tma_load_2d(st + 2 * A_BYTES + A_BYTES, &tm_hi, x, j0 + 128, &full[s]);   //     rows j0+128..j0+255
      tma_load_2d(st + 2 * A_BYTES + B_BYTES, &tm_lo, x, j0, &full[s]);         // B = L
      tma_load_2d(st + 2 * A_BYTES + B_BYTES + A_BYTES, &tm_lo, x, j0 + 128, &full[s]);
      issued = kb + 1;
    }
    // the copies of the last issued k-blocks have landed before this CTA may exit
    for (int kb = issued > ST ? issued - ST : 0; kb < issued; kb++)
      if (!mbar_wait(&full[kb % ST], (uint32_t)((kb / ST) & 1))) *abort_flag = 1;
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    for (int kb = 0; kb < kblocks; kb++) {
      const int s = kb % ST, n = kb / ST;
      if (!mbar_wait(&full[s], (uint32_t)(n & 1))) {
        *abort_flag = 1;
        break;
      }
      if (*abort_flag) break;
      tc_fence_after();
      const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t ah = base, al = base + A_BYTES, bh = base + 2 * A_BYTES, bl = bh + B_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; kk++) {
        const uint32_t off = kk * 32;  // 16 BF16 along K inside the 128-byte swizzled row
        const uint64_t dah = sw128_desc(ah + off), dal = sw128_desc(al + off);
        const uint64_t dbh = sw128_desc(bh + off), dbl = sw128_desc(bl + off);
        umma_bf16(tmem, dah, dbh, (kb | kk) ? 1u : 0u);
        umma_bf16(tmem, dah, dbl, 1u);
        umma_bf16(tmem, dal, dbh, 1u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(accum);
  }
  __syncwarp();

  // ---- epilogue: TMEM lane (32 warp + lane) holds row i0 + 32 warp + lane of the tile ----
  if (!wait_long(accum, 0)) *abort_flag = 1;
  tc_fence_after();
  const int row = i0 + warp * 32 + lane;
  const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
  for (int c0 = 0; c0 < BN; c0 += 16) {
    const int jc = j0 + c0;
    if (jc >= nv) break;                 // warp-uniform
    if (jc + 15 <= i0 + warp * 32) continue;  // no j > row for any row of this warp
    float v[16];
    tmem_ld16(tbase + (uint32_t)c0, v);
#pragma unroll
    for (int t = 0; t < 16; t++) {
      const int j = jc + t;
      if (row < nv && j < nv && row < j) S[(size_t)j * nv + row] = (double)v[t];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, 1);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// H^T and L^T ([nv_pad][k_pad] BF16) from O (ns x nv FP64, row per sample), centred when b and m are given:
// O'(s, k) = O(s, k) - b_s m_k; zero padding
__global__ void split_transpose_kernel(int ns, int nv, const double* __restrict__ O, const double* __restrict__ b,
                                       const double* __restrict__ m, __nv_bfloat16* __restrict__ hiT,
                                       __nv_bfloat16* __restrict__ loT, int k_pad) {
  __shared__ double tile[32][33];
  const int s0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int s = s0 + r, k = k0 + tx;
    double o = (s < ns && k < nv) ? O[(size_t)s * nv + k] : 0.0;
    if (b && s < ns && k < nv) o = fma(-b[s], m[k], o);
    tile[r][tx] = o;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int k = k0 + r, s = s0 + tx;
    const double o = tile[tx][r];
    const __nv_bfloat16 h = __double2bfloat16(o);
    const __nv_bfloat16 l = __double2bfloat16(o - (double)__bfloat162float(h));
    hiT[(size_t)k * k_pad + s] = h;
    loT[(size_t)k * k_pad + s] = l;
  }
}

// exact diagonal: part[c][k] = sum over chunk c of O(s, k)^2; then S(k, k) = sum_c part[c][k]
constexpr int kDiagChunks = 64;
__global__ void colsq_partial(int ns, int nv, const double* __restrict__ O, int chunk, double* __restrict__ part) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (k >= nv) return;
  const int s1 = min(ns, (c + 1) * chunk);
  double a = 0.0;
  for (int s = c * chunk; s < s1; s++) {
    const double o = O[(size_t)s * nv + k];
    a = fma(o, o, a);
  }
  part[(size_t)c * nv + k] = a;
}

__global__ void colsq_finish(int nv, const double* __restrict__ part, double* __restrict__ S) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nv) return;
  double a = 0.0;
  for (int c = 0; c < kDiagChunks; c++) a += part[(size_t)c * nv + k];
  S[(size_t)k * nv + k] = a;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2-D map over a [rows][k_pad] BF16 array with 64 x 128 boxes (128-byte rows) and 128-byte swizzle
bool make_map(CUtensorMap* m, void* base, int k_pad, int rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)k_pad * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, 128};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Padded sizes of the split operands: k_pad = samples rounded up to 64, nv_pad = parameters rounded up to 256.
void rbmpp_bf16x3_pads(int ns, int nv, int* k_pad, int* nv_pad) {
  *k_pad = (ns + BK - 1) / BK * BK;
  *nv_pad = (nv + BN - 1) / BN * BN;
}

// Upper triangle of S = O'^T O' in split-BF16 form, with O' = O - b m^T when b and m are given (else O' = O),
// and the exact FP64 diagonal of O^T O (uncentred).  Column-major nv x nv.
// hi, lo: nv_pad * k_pad BF16 each (16-byte aligned); part: kDiagChunks * nv doubles; d_err: one int,
// set to 1 by a device wait that ran out.  Returns 0, 1 (no tensor-map encoder) or a CUDA error + 100.
int rbmpp_syrk_bf16x3(int ns, int nv, const double* O, const double* b, const double* m, void* hi, void* lo,
                      int* d_err, double* S, double* part, cudaStream_t st) {
  int k_pad = 0, nv_pad = 0;
  rbmpp_bf16x3_pads(ns, nv, &k_pad, &nv_pad);
  CUtensorMap mh, ml;
  if (!make_map(&mh, hi, k_pad, nv_pad) || !make_map(&ml, lo, k_pad, nv_pad)) return 1;
  cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
  if (e) return 100 + (int)e;
  rbmpp_note_launch();
  split_transpose_kernel<<<dim3(k_pad / 32, nv_pad / 32), dim3(32, 8), 0, st>>>(
      ns, nv, O, b, m, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, k_pad);
  if ((e = cudaGetLastError())) return 100 + (int)e;
  if ((e = cudaFuncSetAttribute(syrk_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES)))
    return 100 + (int)e;
  rbmpp_note_launch();
  syrk_bf16x3_kernel<<<dim3(nv_pad / BM, nv_pad / BN), 128, SMEM_BYTES, st>>>(mh, ml, nv, k_pad / BK, S, d_err);
  if ((e = cudaGetLastError())) return 100 + (int)e;
  const int chunk = (ns + kDiagChunks - 1) / kDiagChunks;
  rbmpp_note_launch();
  colsq_partial<<<dim3((nv + 127) / 128, kDiagChunks), 128, 0, st>>>(ns, nv, O, chunk, part);
  rbmpp_note_launch();
  colsq_finish<<<(nv + 255) / 256, 256, 0, st>>>(nv, part, S);
  if ((e = cudaGetLastError())) return 100 + (int)e;
  return 0;
}
