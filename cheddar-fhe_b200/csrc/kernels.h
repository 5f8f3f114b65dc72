// Kernel launch interface shared by the host orchestration (context.cu) and
// the CUDA translation units.  All launches are asynchronous on the given
// stream; all row descriptors travel by value in the kernel parameters, so
// launches need no host-to-device copies and can be captured in CUDA graphs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace chd {

// One limb (N residues of one prime) processed by a batched kernel.
// Constants are plain residues w < q with their Shoup companions
// floor(w 2^32 / q); twiddle tables hold (psi_rev[j], companion) pairs.
struct RowDesc {
  const uint32_t *src;   // input limb
  uint32_t *dst;         // output limb (may equal src for in-place phases)
  const uint32_t *src2;  // second input (ModDown epilogue), or nullptr
  const uint2 *tw;       // twiddle table of this prime (N pairs)
  uint32_t q;            // prime
  uint32_t flags;        // see RowFlags
  int32_t qinv;          // q^-1 mod 2^32 (Montgomery product of kMulSrc2)
  uint32_t pad_;
  uint32_t c0, c0s;      // pre-multiplier (forward) / output constant (inverse)
  uint32_t c1, c1s;      // ModDown epilogue: src2 padding multiplier
  uint32_t c2, c2s;      // ModDown epilogue: (prod of dropped primes)^-1
};

enum RowFlags : uint32_t {
  kPreMult = 1u,       // forward NTT: multiply input by c0 first
  kCentre = 2u,        // inverse NTT: write the centred representative
  kHasSrc2 = 4u,       // ModDown epilogue: src2 exists for this row
  kPadSrc2 = 8u,       // ModDown epilogue: multiply src2 by c1 first
  kModDownEpi = 16u,   // forward NTT row phase: apply (src2*c1 - x) * c2
  kMulSrc2 = 32u,      // inverse NTT row phase: input is src (.) src2 (Montgomery)
};

// rows per row-phase launch: 256 descriptors of 72 bytes keep the launch
// parameters under the 32 KiB limit
constexpr int kMaxRows = 256;

struct RowBatch {
  int count;
  RowDesc rows[kMaxRows];
};
static_assert(sizeof(RowBatch) + 16 <= 32764, "row batch beyond the kernel parameter limit");

// Forward negacyclic NTT (bit-reversed output) of `count` limbs.
// Column phase then row phase for log_n = 16; a single-kernel shared-memory
// transform for log_n <= 15.  In-place allowed (dst == src).
void launch_ntt_fwd(const RowBatch &rb, int log_n, cudaStream_t s);
// Row phase only / column phase only (used by fused pipelines and tests)
void launch_ntt_fwd_cols(const RowBatch &rb, int log_n, cudaStream_t s);
void launch_ntt_fwd_rows(const RowBatch &rb, int log_n, cudaStream_t s);
// Inverse NTT (bit-reversed input); epilogue x * c0, canonical or centred
// (kCentre).  tw must point at the inverse twiddle table.
void launch_ntt_inv(const RowBatch &rb, int log_n, cudaStream_t s);

// Base conversion of one job: out[m][n] = (sum_k xt[k][n] * T[m][k]) * 2^-32
// mod p_m.  xt holds K consecutive centred limbs; destination limb m is
// row out_row[m] of `out` and uses the prime of global index out_gidx[m].
struct BConvJob {
  const int32_t *xt;
  uint32_t *out;
  const int32_t *table;  // device [M][K] centred constants
  int K, M;
  uint8_t out_row[64];
  uint8_t out_gidx[64];
};
constexpr int kMaxBConvJobs = 24;
struct BConvBatch {
  int count;
  const uint32_t *primes;  // device table of all primes (by global index)
  const int32_t *qinvs;
  BConvJob jobs[kMaxBConvJobs];
};
void launch_bconv(const BConvBatch &b, int log_n, cudaStream_t s);

// BConv of npoly polynomials on the tcgen05 tensor cores (bconv_tc.cu):
// xt [npoly][K][n] centred sources, out [npoly][M][n]; bmat is the B operand
// (bytes of 2^(8j) T[m][k] mod p_m) in the canonical K-major shared-memory
// image, ksteps x nb x 32 bytes.  err is set to 1 when an MMA completion wait
// runs out (the kernel then returns without finishing).
struct BConvTcDesc {
  const int32_t *xt;
  uint32_t *out;
  const uint8_t *bmat;
  int *err;
  int K, M, n, npoly;
  int ksteps;      // ceil(4K / 32)
  int nb;          // 4M rounded up to a multiple of 16 (MMA N)
  int tpi;         // 128-row tiles per CTA iteration (1, 2 or 4), each with nb TMEM columns
  int tmem_cols;   // power of two >= max(32, 2 * tpi * nb) (two accumulator buffers), <= 512
  uint32_t idesc;  // tcgen05 instruction descriptor (kind::i8, s8 x u8 -> s32, M = 128, N = nb)
  // test hook, 0 in normal use: > 0 makes each CTA's first accumulator wait
  // poll an mbarrier that nothing signals, this many times, so that the
  // bounded wait runs out and the give-up path (error word, drain of the
  // MMAs in flight, TMEM release) runs
  uint32_t stall_polls;
  uint32_t p[64];
  int32_t pinv[64];
};
size_t bconv_tc_smem(int tpi, int ksteps, int nb);
int launch_bconv_tc(const BConvTcDesc &d, int num_sms, cudaStream_t s);

// ---- bootstrapping kernels (boot_kernels.cu) ----
// Lift of a level -1 polynomial (coefficient domain, nbase = 1 or 2 base
// limbs per part) to the rows primes p[] (kernel::ModUpToMax1/2).
struct ModUpToMaxDesc {
  const uint32_t *src[2];  // per part: [nbase][n]
  uint32_t *dst[2];        // per part: [rows][n]
  uint32_t p[64];
  uint32_t q0, q1;
  int nbase, rows, parts, n;
};
void launch_modup_to_max(const ModUpToMaxDesc &d, cudaStream_t s);

// out_(b, a)[c][o][r] = sum_t pt[o][t][r] (.) in_(b, a)[c][t][r] over the
// (o, t) pairs with a plaintext (pt[o][t] == nullptr: no term).  Up to
// kMaxPtAccumCts ciphertexts share the plaintexts.
constexpr int kMaxPtAccumIn = 64;
constexpr int kMaxPtAccumOuts = 16;
constexpr int kMaxPtAccumCts = 8;
struct PtAccumDesc {
  const uint32_t *in_b[kMaxPtAccumCts][kMaxPtAccumIn], *in_a[kMaxPtAccumCts][kMaxPtAccumIn];
  uint32_t *out_b[kMaxPtAccumCts][kMaxPtAccumOuts], *out_a[kMaxPtAccumCts][kMaxPtAccumOuts];
  const uint32_t *pt[kMaxPtAccumOuts][kMaxPtAccumIn];
  uint32_t q[64];
  int32_t qinv[64];
  int rows, ins, outs, n, count;
};
// tune: time the 3- and 4-CTA forms of the 4-output kernel on the first
// launch of each shape and keep the faster
void launch_pt_accum(const PtAccumDesc &d, cudaStream_t s, bool tune = false);

// dst[o][r] = sum_t c[t][r] * src[t][o][src_row0[t] + r] for every output o
// (a ciphertext part; several ciphertexts sharing the terms' constants fill
// one launch); a null src[t][o] leaves term t out of output o
constexpr int kMaxConstAccumTerms = 16;
constexpr int kMaxConstAccumOuts = 24;
struct ConstAccumDesc {
  const uint32_t *src[kMaxConstAccumTerms][kMaxConstAccumOuts];
  int src_row0[kMaxConstAccumTerms];
  uint32_t c[kMaxConstAccumTerms][64];
  uint32_t *dst[kMaxConstAccumOuts];
  uint32_t q[64];
  int32_t qinv[64];
  int terms, rows, parts, n;  // parts: the number of outputs
};
void launch_const_accum(const ConstAccumDesc &d, cudaStream_t s);

// Fused ModSwitch column pass (N = 2^16 only): per 16-column tile
//   x~_k  = centre(INTT column phase(src_k) * c0_k)        (K <= 16 sources)
//   y_m   = (sum_k x~_k T[m][k]) * 2^-32 mod p_m           (exact BConv)
//   dst_m = NTT column phase(y_m)                          (lazy [0, 2q))
// src_k = src + src_row[k] * N holds the INTT row-phase output; dst_m =
// dst + dst_row[m] * N is finished by launch_ntt_fwd_rows.
struct MSColJob {
  const uint32_t *src;
  uint32_t *dst;
  const int32_t *table;  // device [M][K]
  int K, M;
  uint8_t src_row[16], src_gidx[16];
  uint8_t dst_row[64], dst_gidx[64];
  uint32_t c0[16], c0s[16];
};
// jobs per column-pass launch: 64 descriptors of 320 bytes keep the launch
// parameters under the 32 KiB limit (a batched ModDown of 30 ciphertexts'
// 60 polynomials is one launch per stream half)
constexpr int kMaxMSColJobs = 64;
struct MSColBatch {
  int count;
  int engine;             // base conversion on 0: CUDA cores, 1: tensor cores, 3: tensor cores with
                          // 256-thread tiles (K <= 12; larger K runs engine 1); 4 (autotuner only):
                          // 3 with the K <= 8 kernel sized for 2 CTAs per SM
  int *err;               // set to 1 when a tensor-core wait gives up
  const uint2 *tw, *itw;  // twiddle tables [nprimes][N]
  const uint32_t *primes;
  const int32_t *qinvs;
  MSColJob jobs[kMaxMSColJobs];
};
static_assert(sizeof(MSColBatch) + 16 <= 32764, "column-pass batch beyond the kernel parameter limit");
void launch_modswitch_cols(const MSColBatch &b, int log_n, cudaStream_t s);
// the autotuned choices (engine, target split) cached so far: 6 ints per
// shape (device, largest K, jobs, largest M, engine, split); returns the count
int modswitch_tuned_shapes(int *out, int cap);
// tensor-core column pass (modswitch_tc.cu); every job has K <= 16
void launch_modswitch_cols_tc(const MSColBatch &b, int max_k, cudaStream_t s);
size_t modswitch_cols_tc_smem(int kmax);
// the same on 256-thread tiles, 8 coefficients per thread (modswitch_tc8.cu),
// for jobs with K <= 12; regs128 sizes the K <= 8 kernel for 2 CTAs per SM
// (128 registers) instead of 3 (80)
bool modswitch_cols_tc8_supports(int max_k);
void launch_modswitch_cols_tc8(const MSColBatch &b, int max_k, bool regs128, cudaStream_t s);
void launch_ntt_inv_rows(const RowBatch &rb, int log_n, cudaStream_t s);

// Fused key-switching row pass (N = 2^16), see keyswitch.cu.  Modes:
//   0 HMult:       own ModUp value a1 a2, d0 = b1 b2, d1 = b1 a2 + a1 b2
//   1 MultKey:     own ModUp value a1 (= ax), d0 = b1 (= bx)
//   2 Relinearize: own ModUp value a2 (= rx), d0 = b1 (= bx), d1 = a1 (= ax)
struct KSRowsCt {
  const uint32_t *mu[8];             // ModUp column-pass outputs [tot][N] per digit
  const uint32_t *b1, *a1, *b2, *a2; // inputs [nq][N]
  uint32_t *acc_b, *acc_a;           // kept primes: evaluation-domain accumulators [tot][N]
  uint32_t *drop_b, *drop_a;         // dropped primes: INTT row-phase output [ndrop][N]
  int lv;                            // entry of KSRowsDesc::lv describing its level
};
// Row tables of one level of the extended basis Q u P (row j of a
// ciphertext at that level); several levels can share one launch.
struct KSRowsLevel {
  const uint32_t *kb[8], *ka[8];     // key digit pointers (row 0 of the key basis)
  int beta, rows, nq;
  int16_t key_row[64];
  uint8_t gidx[64];
  int8_t own_digit[64];              // digit owning row j (q primes), else -1
  int8_t drop_idx[64];               // row of j in the drop buffers, else -1
  uint32_t p_prod[64];               // Montgomery P mod q_j (q rows)
};
constexpr int kMaxKSRowsCts = 16;
constexpr int kMaxKSRowsLevels = 8;
struct KSRowsDesc {
  const uint2 *tw, *itw;
  const uint32_t *primes;            // [nprimes] by global index
  const int32_t *qinvs;
  int count, mode, nlv, max_rows;
  KSRowsLevel lv[kMaxKSRowsLevels];
  KSRowsCt ct[kMaxKSRowsCts];
};
// tune: pick the row-pass variant per launch shape by timing both once
// (the context's CHD_BCONV_AUTO); otherwise the one without prefetching
void launch_ks_rows(const KSRowsDesc &d, int log_n, cudaStream_t s, bool tune = false);
// the row-pass choices cached so far: 5 ints per shape (device, ciphertexts,
// largest row count, mode, prefetching variant); returns the count
int ks_rows_tuned_shapes(int *out, int cap);

// Key-switching inner product with the P * (d0, d1) term folded in:
//   acc_b[r] = sum_i mu_i[r] * kb_i[r] + (r < nq ? p_prod[r] * d0[r] : 0)
//   acc_a[r] = sum_i mu_i[r] * ka_i[r] + (r < nq && d1 ? p_prod[r] * d1[r] : 0)
// for up to kMaxKeyMacCts ciphertexts sharing one key (the ciphertext is the
// fastest-varying part of grid.x, so the key tile is shared through L2).
constexpr int kMaxKeyMacCts = 16;
struct KeyMacCt {
  const uint32_t *mu[8];     // beta ModUp outputs, each [rows][N]
  const uint32_t *d0, *d1;   // [nq][N] or nullptr
  uint32_t *acc_b, *acc_a;   // [rows][N]
};
struct KeyMacDesc {
  const uint32_t *kb[8];     // key bx of digit i, row-0 pointer of the key basis
  const uint32_t *ka[8];
  uint32_t q[64];
  int32_t qinv[64];
  uint32_t p_prod[64];       // Montgomery P mod q, q rows only
  int16_t key_row[64];       // key basis row of accumulator row r
  int beta, rows, nq, count;
  KeyMacCt ct[kMaxKeyMacCts];
};
void launch_key_mac(const KeyMacDesc &d, int log_n, cudaStream_t s);

// Element-wise kernels over a list of limbs (same op for every limb).
enum class ElemOp : int {
  kAdd, kSub, kNeg, kMult, kAddConst, kSubConst, kSubOppConst, kMultConst,
  kCopy, kMultImagUnit, kMultAdd, kMultConstAdd
};
struct ElemRow {
  const uint32_t *a, *b;  // inputs (b unused for unary)
  const uint32_t *c;      // accumulator input for kMultAdd / kMultConstAdd
  uint32_t *dst;
  uint32_t q;
  int32_t qinv;
  uint32_t k;             // per-limb constant
};
// limbs per element-wise launch: every part of a ciphertext of up to 64
// primes, or of a few of them, in one launch (parameter size checked below)
constexpr int kMaxElemRows = 256;
struct ElemBatch {
  int count;
  ElemRow rows[kMaxElemRows];
};
static_assert(sizeof(ElemBatch) + 16 <= 32764, "element-wise batch beyond the kernel parameter limit");
void launch_elementwise(ElemOp op, const ElemBatch &b, int log_n, cudaStream_t s);

// Tensor product of (b1, a1) x (b2, a2) -> (d0, d1, d2) (Karatsuba form)
struct TensorRow {
  const uint32_t *b1, *a1, *b2, *a2;
  uint32_t *d0, *d1, *d2;
  uint32_t q;
  int32_t qinv;
};
struct TensorBatch {
  int count;
  TensorRow rows[64];
};
void launch_tensor(const TensorBatch &b, int log_n, cudaStream_t s);

// Automorphism X -> X^g in the bit-reversed evaluation domain (gather):
// dst[k] = src[brev(((2 brev(k) + 1) g - 1) mod 2N)]
// dst = Permute(src (+ src2)) (+ add), one limb per row
struct PermuteRow {
  const uint32_t *src;
  const uint32_t *src2;  // optional second source, added before the gather
  uint32_t *dst;
  const uint32_t *add;   // optional addend (PermuteAccum with src0)
  uint32_t q;
};
constexpr int kMaxPermuteRows = 256;
struct PermuteBatch {
  int count;
  uint32_t galois;
  PermuteRow rows[kMaxPermuteRows];
};
static_assert(sizeof(PermuteBatch) + 16 <= 32764, "permute batch beyond the kernel parameter limit");
void launch_permute(const PermuteBatch &b, int log_n, cudaStream_t s);

// Hoisted rotations: one launch for up to kMaxHoist rotations of one ModUp'ed
// input.  For every rotation j and row r of the extended basis Q u P:
//   v = sum_i mu_i[r] (.) key_j,i[r]  (+ P * bx[r] on q rows for the b part)
// scattered through the automorphism: out_j[galois_src(k, g_j)] = v[k] with
// g_j the Galois factor of N/2 - r_j (the inverse of rotation r_j).
constexpr int kMaxHoist = 32;
constexpr int kMaxHoistCts = 8;  // ciphertexts sharing the keys of one launch
struct HoistDesc {
  const uint32_t *mu[kMaxHoistCts][8];
  const uint32_t *bxp[kMaxHoistCts];     // P * bx on q rows, [nq][N]
  const uint32_t *kb[kMaxHoist][8];      // key row-0 pointers per rotation/digit
  const uint32_t *ka[kMaxHoist][8];
  uint32_t *out_b[kMaxHoistCts][kMaxHoist];  // outputs [rows][N]
  uint32_t *out_a[kMaxHoistCts][kMaxHoist];
  uint32_t galois_inv[kMaxHoist];
  uint32_t q[64];
  int32_t qinv[64];
  int16_t key_row[64];
  int beta, rows, nq, R, count;
};
// tune: time the 3- and 4-CTA forms on the first launch of each shape (up
// to 4 digits) and keep the faster
void launch_hoisted(const HoistDesc &d, int log_n, cudaStream_t s, bool tune = false);

}  // namespace chd
