// GPU pin driver: runs the reference's own Montgomery primitives
// (include/common/Basic.cuh:80-88, 120-125, 150-157, 251-260 — compiled from
// the reference tree for sm_100a) on a fixed, in-bounds batch of operands
// and writes the raw results to a binary file.  tests/test_oracle_pins.py
// compares them with the oracle's restatement.  Test infrastructure only.
//
// File format (little endian): u32 count, then count records of
//   u32 q, i32 q_inv, i32 a, i32 b, i32 lazy_mult, u32 mult_mont,
//   u32 reduce_of_wide, i32 normalize_a
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "common/Basic.cuh"

using namespace cheddar;

struct Rec {
  uint32_t q;
  int32_t q_inv;
  int32_t a, b;
  int32_t lazy;
  uint32_t mont;
  uint32_t red;
  int32_t norm;
};

__global__ void pin_kernel(Rec *r, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rec x = r[i];
  x.lazy = basic::detail::__mult_montgomery_lazy<uint32_t>(x.a, x.b, x.q, x.q_inv);
  uint32_t ua = static_cast<uint32_t>(x.a < 0 ? x.a + static_cast<int32_t>(x.q) : x.a);
  uint32_t ub = static_cast<uint32_t>(x.b < 0 ? x.b + static_cast<int32_t>(x.q) : x.b);
  x.mont = basic::MultMontgomery<uint32_t>(ua, ub, x.q, x.q_inv);
  int64_t wide = static_cast<int64_t>(x.a) * static_cast<int64_t>(x.b);
  x.red = basic::ReduceMontgomery<uint32_t>(wide, x.q, x.q_inv);
  x.norm = basic::Normalize<uint32_t>(ua, x.q);
  r[i] = x;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s out.bin prime...\n", argv[0]);
    return 2;
  }
  std::vector<Rec> recs;
  unsigned long long s = 0x243f6a8885a308d3ull;
  auto next = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
  };
  for (int a = 2; a < argc; a++) {
    uint32_t q = static_cast<uint32_t>(std::strtoul(argv[a], nullptr, 10));
    // q^-1 mod 2^32 by Newton iteration (q odd)
    uint32_t inv = q;
    for (int k = 0; k < 5; k++) inv *= 2u - q * inv;
    for (int k = 0; k < 4096; k++) {
      Rec r{};
      r.q = q;
      r.q_inv = static_cast<int32_t>(inv);
      // operands in (-q, q): the documented input range of the lazy product
      int64_t a1 = static_cast<int64_t>(next() % (2ull * q - 1)) - (q - 1);
      int64_t b1 = static_cast<int64_t>(next() % (2ull * q - 1)) - (q - 1);
      if (k < 8) {  // edge operands
        int64_t e[8] = {0, 1, -1, static_cast<int64_t>(q) - 1, -(static_cast<int64_t>(q) - 1),
                        static_cast<int64_t>(q >> 1), -static_cast<int64_t>(q >> 1), 2};
        a1 = e[k];
        b1 = e[7 - k];
      }
      r.a = static_cast<int32_t>(a1);
      r.b = static_cast<int32_t>(b1);
      recs.push_back(r);
    }
  }
  int n = static_cast<int>(recs.size());
  Rec *d = nullptr;
  if (cudaMalloc(&d, sizeof(Rec) * n) != cudaSuccess) return 1;
  cudaMemcpy(d, recs.data(), sizeof(Rec) * n, cudaMemcpyHostToDevice);
  pin_kernel<<<(n + 255) / 256, 256>>>(d, n);
  if (cudaDeviceSynchronize() != cudaSuccess) return 1;
  cudaMemcpy(recs.data(), d, sizeof(Rec) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 1;
  uint32_t cnt = static_cast<uint32_t>(n);
  std::fwrite(&cnt, 4, 1, f);
  std::fwrite(recs.data(), sizeof(Rec), n, f);
  std::fclose(f);
  return 0;
}
