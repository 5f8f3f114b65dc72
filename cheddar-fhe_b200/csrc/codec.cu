// Encoder and decoder on the device.
//
// Encode (src/core/Encode.cpp:23-41, 84-107, 135-190 of the reference):
// complex slots -> special IFFT in FP64 -> times the scale, truncated toward
// zero to an integer -> residues of the level's primes -> NTT with the
// Montgomery conversion.  Decode (Encode.cpp:45-70, 109-133, 192-248):
// INTT times (N q-hat_i)^-1 -> CRT to the centred integer -> double / scale
// -> special FFT.
//
// The FP64 steps are the reference's operations in the reference's order,
// each rounded once (complex products as (ac - bd, ad + bc) with separately
// rounded products, the form GCC emits for std::complex<double>; no fused
// multiply-add), so the device results are bit-identical to the reference's
// host encoder and decoder.  The integer conversions follow its bigint
// backend (BigInt_tommath.cpp over libtommath): truncation toward zero on
// the way in, and on the way out the centred integer converted to double by
// folding its 60-bit digits from the most significant one down.
#include <cmath>
#include <complex>

#include "host.h"
#include "kernels.h"

namespace chd {
namespace {

__device__ __forceinline__ double2 dadd2(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 dsub2(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
// (a + bi)(c + di) = (ac - bd) + (ad + bc) i, every product and sum rounded
__device__ __forceinline__ double2 cmul(double2 y, double2 t) {
  return make_double2(__dsub_rn(__dmul_rn(y.x, t.x), __dmul_rn(y.y, t.y)),
                      __dadd_rn(__dmul_rn(y.x, t.y), __dmul_rn(y.y, t.x)));
}

// One stage of Encoder::SpecialIFFT (Encode.cpp:84-107): butterflies at
// distance `stride`, twiddle index (st8 - (5^j mod 2N) mod st8) * gap
__global__ void k_special_ifft_stage(double2 *d, int ns, int stride, const double2 *tw, const int *galois, int M) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns / 2) return;
  const int j = b % stride, i = (b / stride) * 2 * stride;
  const int st8 = stride << 3, gap = M / st8;
  const int ti = (st8 - galois[j] % st8) * gap;
  const double2 u = d[i + j], v = d[i + j + stride];
  d[i + j] = dadd2(u, v);
  d[i + j + stride] = cmul(dsub2(u, v), tw[ti]);
}

// One stage of Encoder::SpecialFFT (Encode.cpp:109-133)
__global__ void k_special_fft_stage(double2 *d, int ns, int stride, const double2 *tw, const int *galois, int M) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns / 2) return;
  const int j = b % stride, i = (b / stride) * 2 * stride;
  const int st8 = stride << 3, gap = M / st8;
  const int ti = (galois[j] % st8) * gap;
  const double2 x = d[i + j], y = cmul(d[i + j + stride], tw[ti]);
  d[i + j] = dadd2(x, y);
  d[i + j + stride] = dsub2(x, y);
}

// BitReverseVector (include/common/CommonUtils.h), out of place
__global__ void k_bit_reverse(const double2 *src, double2 *dst, int ns, int lb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  dst[__brev(static_cast<unsigned>(i)) >> (32 - lb)] = src[i];
}

// round-toward-zero integer of v reduced to [0, p) (BigInt(double) then
// BigInt::Mod): exact for every finite double
__host__ __device__ __forceinline__ uint32_t trunc_mod_dev(double v, uint32_t p) {
  if (v == 0.0) return 0;
  const bool neg = v < 0;
  const double a = fabs(v);
  uint64_t r;
  if (a < 18446744073709551616.0) {
    r = static_cast<uint64_t>(a) % p;
  } else {
    int e;
    const double m = frexp(a, &e);  // a = m 2^e, m in [0.5, 1)
    const uint64_t mi = static_cast<uint64_t>(ldexp(m, 53));
    uint64_t pw = 1 % p, b = 2;
    for (int sh = e - 53; sh; sh >>= 1) {
      if (sh & 1) pw = pw * b % p;
      b = b * b % p;
    }
    r = (mi % p) * pw % p;
  }
  if (neg && r) r = p - r;
  return static_cast<uint32_t>(r);
}

// Encode.cpp:84-107 tail and 135-190: slot i of the bit-reversed IFFT output,
// divided by ns and times the scale, truncated; residues at coefficient
// i * gap (real part) and i * gap + N/2 (imaginary part) of every prime row
struct EncodeRows {
  uint32_t p[64];
  int rows;
};
__global__ void k_encode_residues(const double2 *d, int ns, double scale, const __grid_constant__ EncodeRows er,
                                  uint32_t *mx, int n, int gap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const double dn = static_cast<double>(ns);
  const double re = __dmul_rn(__ddiv_rn(d[i].x, dn), scale);
  const double im = __dmul_rn(__ddiv_rn(d[i].y, dn), scale);
  const int k = blockIdx.y;
  const uint32_t p = er.p[k];
  uint32_t *row = mx + static_cast<size_t>(k) * n;
  row[i * gap] = trunc_mod_dev(re, p);
  row[i * gap + n / 2] = trunc_mod_dev(im, p);
}

// Encode.cpp:192-248 (PlaintextToComplexVector): the centred CRT integer
// X = sum_j y_j q-hat_j mod Q of each used coefficient, as a double divided
// by the scale.  With k = round(sum_j y_j / q_j), X = sum_j y_j q-hat_j - k Q
// exactly, computed modulo 2^128 (|X| < 2^127 for any decryptable value).
struct CrtRows {
  uint32_t q[64];
  uint64_t qhat_lo[64], qhat_hi[64];
  uint64_t Q_lo, Q_hi;
  int rows;
};
__device__ __forceinline__ void mac128(uint64_t &lo, uint64_t &hi, uint64_t a, uint64_t blo, uint64_t bhi) {
  const uint64_t plo = a * blo, phi = __umul64hi(a, blo) + a * bhi;
  lo += plo;
  hi += phi + (lo < plo ? 1u : 0u);
}
__device__ double crt_value(const uint32_t *y, size_t stride, const CrtRows &cr) {
  double s = 0.0;
  uint64_t lo = 0, hi = 0;
  for (int j = 0; j < cr.rows; j++) {
    const uint32_t v = y[j * stride];
    s = __dadd_rn(s, __ddiv_rn(static_cast<double>(v), static_cast<double>(cr.q[j])));
    mac128(lo, hi, v, cr.qhat_lo[j], cr.qhat_hi[j]);
  }
  const uint64_t k = static_cast<uint64_t>(floor(s + 0.5));
  // X = S - k Q mod 2^128
  const uint64_t klo = k * cr.Q_lo, khi = __umul64hi(k, cr.Q_lo) + k * cr.Q_hi;
  uint64_t xlo = lo - klo;
  uint64_t xhi = hi - khi - (lo < klo ? 1u : 0u);
  const bool neg = (xhi >> 63) != 0;
  if (neg) {  // magnitude of the two's complement value
    xlo = ~xlo + 1;
    xhi = ~xhi + (xlo == 0 ? 1u : 0u);
  }
  // 60-bit digits, folded from the most significant: d = d 2^60 + digit
  const uint64_t m60 = (uint64_t{1} << 60) - 1;
  const uint64_t d0 = xlo & m60;
  const uint64_t d1 = ((xlo >> 60) | (xhi << 4)) & m60;
  const uint64_t d2 = xhi >> 56;
  const double fac = 1152921504606846976.0;  // 2^60
  double d = 0.0;
  if (d2) d = __ull2double_rn(d2);
  if (d2 || d1) d = __dadd_rn(__dmul_rn(d, fac), __ull2double_rn(d1));
  d = __dadd_rn(__dmul_rn(d, fac), __ull2double_rn(d0));
  return neg ? -d : d;
}
__global__ void k_crt_decode(const uint32_t *y, int n, int gap, int ns, double scale,
                             const __grid_constant__ CrtRows cr, double2 *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const double re = crt_value(y + static_cast<size_t>(i) * gap, n, cr);
  const double im = crt_value(y + static_cast<size_t>(i) * gap + n / 2, n, cr);
  out[i] = make_double2(__ddiv_rn(re, scale), __ddiv_rn(im, scale));
}

int log2_exact(int x) {
  int lb = 0;
  while ((1 << lb) < x) lb++;
  return lb;
}

}  // namespace

Status Context::codec_tables() {
  if (d_enc_tw) return kOk;
  const auto &tw = enc_twiddles();
  CHD_CHECK(cudaMalloc(&d_enc_tw, tw.size() * sizeof(double2)) == cudaSuccess, kErrAlloc,
            "encoder: twiddle table allocation failed");
  CHD_CHECK(cudaMalloc(&d_galois, P->galois.size() * sizeof(int)) == cudaSuccess, kErrAlloc,
            "encoder: galois table allocation failed");
  cudaMemcpy(d_enc_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice);
  cudaMemcpy(d_galois, P->galois.data(), P->galois.size() * sizeof(int), cudaMemcpyHostToDevice);
  return check_cuda("encoder tables");
}

Status Context::encode(int level, double scale, const std::complex<double> *msg, int msg_len, int num_aux,
                       uint32_t *pt_dev, int *num_slots_out) {
  // Encoder::Encode / EncodeWorker / ComplexVectorToPlaintext,
  // Encode.cpp:23-41, 84-107, 135-190, on the device
  CHD_CHECK(msg_len >= 1 && msg_len <= P->n / 2, kErrInvalidArg, "Encode: 1 <= message length <= N/2");
  CHD_CHECK(num_aux >= 0 && num_aux <= P->alpha, kErrInvalidArg, "Encode: invalid number of aux primes");
  CHD_CHECK(level >= -1 && level <= P->max_level, kErrInvalidLevel, "Encode: invalid level");
  CHD_TRY(codec_tables());
  int ns = 1;
  while (ns < msg_len) ns *= 2;
  const NP np = P->level_np(level, num_aux);
  const int tot = np.total(), n = P->n, gap = n / 2 / ns, M = 2 * n;
  CHD_CHECK(tot <= 64, kErrUnsupported, "Encode: more than 64 primes");
  ArenaScope scope(arena);
  double2 *d = static_cast<double2 *>(arena.alloc(2 * static_cast<size_t>(ns) * sizeof(double2)));
  CHD_CHECK(d, kErrAlloc, "Encode: scratch allocation failed");
  double2 *e = d + ns;
  std::vector<double2> h(ns, make_double2(0.0, 0.0));
  for (int i = 0; i < msg_len; i++) h[i] = make_double2(msg[i].real(), msg[i].imag());
  cudaMemcpyAsync(d, h.data(), ns * sizeof(double2), cudaMemcpyHostToDevice, stream);
  const int th = 256;
  for (int stride = ns / 2; stride >= 1; stride /= 2)
    k_special_ifft_stage<<<(ns / 2 + th - 1) / th, th, 0, stream>>>(d, ns, stride, d_enc_tw, d_galois, M);
  k_bit_reverse<<<(ns + th - 1) / th, th, 0, stream>>>(d, e, ns, log2_exact(ns));
  if (gap > 1) cudaMemsetAsync(pt_dev, 0, static_cast<size_t>(tot) * n * 4, stream);
  EncodeRows er{};
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  for (int k = 0; k < tot; k++) er.p[k] = P->primes[g[k]];
  er.rows = tot;
  k_encode_residues<<<dim3((ns + th - 1) / th, tot), th, 0, stream>>>(e, ns, scale, er, pt_dev, n, gap);
  if (num_slots_out) *num_slots_out = ns;
  // NTT(..., true): to the evaluation domain, Montgomery form
  CHD_TRY(ntt(np, pt_dev, true));
  // the host message buffer must outlive its upload
  return cudaStreamSynchronize(stream) == cudaSuccess ? kOk : check_cuda("encode");
}

Status Context::decode(int level, double scale, const uint32_t *pt_dev, int num_slots, std::complex<double> *out) {
  // Encoder::Decode, Encode.cpp:45-70, 109-133, 192-248, on the device
  CHD_CHECK(level >= -1 && level <= P->max_level, kErrInvalidLevel, "Decode: invalid level");
  CHD_CHECK(num_slots >= 1 && num_slots <= P->n / 2 && (num_slots & (num_slots - 1)) == 0, kErrInvalidArg,
            "Decode: the slot count must be a power of two <= N/2");
  CHD_TRY(codec_tables());
  const NP np = P->level_np(level);
  const int tot = np.q(), n = P->n, gap = n / 2 / num_slots, M = 2 * n;
  CHD_CHECK(tot <= 64, kErrUnsupported, "Decode: more than 64 primes");
  std::vector<int> g(tot);
  P->gidx(np, g.data());
  // INTTAndMultConst with (N prod_{j != i} q_j)^-1, applied like a Montgomery
  // constant (the plaintext carries the Montgomery factor), Encode.cpp:52-68
  ArenaScope scope(arena);
  uint32_t *y = static_cast<uint32_t *>(arena.alloc(static_cast<size_t>(tot) * n * 4));
  double2 *d = static_cast<double2 *>(arena.alloc(2 * static_cast<size_t>(num_slots) * sizeof(double2)));
  CHD_CHECK(y && d, kErrAlloc, "Decode: scratch allocation failed");
  double2 *e = d + num_slots;
  std::vector<RowDesc> rows;
  CrtRows cr{};
  unsigned __int128 Q = 1;
  for (int i = 0; i < tot; i++) {
    const uint32_t q = P->primes[g[i]];
    uint32_t c = static_cast<uint32_t>(n % q);
    unsigned __int128 qhat = 1;
    for (int j = 0; j < tot; j++)
      if (j != i) {
        c = prime::mul_mod(c, P->primes[g[j]], q);
        qhat *= P->primes[g[j]];
      }
    RowDesc r{};
    r.src = pt_dev + static_cast<size_t>(i) * n;
    r.dst = y + static_cast<size_t>(i) * n;
    r.tw = itw(g[i]);
    r.q = q;
    mont_as_shoup(prime::inv_mod(c, q), g[i], &r.c0, &r.c0s);
    rows.push_back(r);
    cr.q[i] = q;
    cr.qhat_lo[i] = static_cast<uint64_t>(qhat);
    cr.qhat_hi[i] = static_cast<uint64_t>(qhat >> 64);
    Q *= q;
  }
  cr.Q_lo = static_cast<uint64_t>(Q);
  cr.Q_hi = static_cast<uint64_t>(Q >> 64);
  cr.rows = tot;
  for_row_batches(rows, [&](const RowBatch &rb) { launch_ntt_inv(rb, P->log_n, stream); });
  const int th = 256;
  k_crt_decode<<<(num_slots + th - 1) / th, th, 0, stream>>>(y, n, gap, num_slots, scale, cr, d);
  k_bit_reverse<<<(num_slots + th - 1) / th, th, 0, stream>>>(d, e, num_slots, log2_exact(num_slots));
  for (int stride = 1; stride < num_slots; stride *= 2)
    k_special_fft_stage<<<(num_slots / 2 + th - 1) / th, th, 0, stream>>>(e, num_slots, stride, d_enc_tw, d_galois,
                                                                           M);
  static_assert(sizeof(std::complex<double>) == sizeof(double2), "complex layout");
  cudaMemcpyAsync(out, e, num_slots * sizeof(double2), cudaMemcpyDeviceToHost, stream);
  return cudaStreamSynchronize(stream) == cudaSuccess ? kOk : check_cuda("decode");
}

}  // namespace chd
