// Pin driver: compiles the reference's own host prime utilities
// (include/common/PrimeUtils.h), its Normalize (include/common/Basic.cuh:229)
// and its BitReverseVector (include/common/CommonUtils.h) straight from the
// reference tree, and prints, for every prime given on the command line:
//   prime, generator, psi (primitive 2N-th root), psi^-1, q^-1 mod 2^32,
//   N^-1, R^2 mod q, and a short hash of the bit-reversed Montgomery twiddle
//   tables built the way NTTHandler::PopulateTwiddleFactors
//   (src/core/NTT.cu:1233-1299) builds them.
// Output is one JSON object per line; tests/golden/make_golden.py turns it
// into a fixture.  This file is test infrastructure, not product code.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "common/Basic.cuh"
#include "common/CommonUtils.h"
#include "common/PrimeUtils.h"

using namespace cheddar;

static unsigned long long fnv(const std::vector<uint32_t> &v) {
  unsigned long long h = 1469598103934665603ull;
  for (uint32_t x : v) {
    for (int b = 0; b < 4; b++) {
      h ^= (x >> (8 * b)) & 0xff;
      h *= 1099511628211ull;
    }
  }
  return h;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s log_degree prime...\n", argv[0]);
    return 2;
  }
  int log_degree = std::atoi(argv[1]);
  int degree = 1 << log_degree;
  for (int a = 2; a < argc; a++) {
    uint32_t p = static_cast<uint32_t>(std::strtoul(argv[a], nullptr, 10));
    uint32_t g = primeutil::FindGenerator<uint32_t>(p);
    uint32_t psi = primeutil::FindPrimitiveMthRoot<uint32_t>(2 * degree, p);
    uint32_t psi_inv = primeutil::InvMod<uint32_t>(psi, p);
    int32_t qinv = primeutil::InvModBase<uint32_t>(p);
    uint32_t n_inv = primeutil::InvMod<uint32_t>(degree, p);
    uint32_t r2 = primeutil::ToMontgomery(primeutil::ToMontgomery<uint32_t>(1, p), p);
    std::vector<uint32_t> psi_rev(degree), psi_inv_rev(degree);
    psi_rev[0] = 1;
    psi_inv_rev[0] = 1;
    for (int j = 1; j < degree; j++) {
      psi_rev[j] = primeutil::MultMod(psi_rev[j - 1], psi, p);
      psi_inv_rev[j] = primeutil::MultMod(psi_inv_rev[j - 1], psi_inv, p);
    }
    BitReverseVector(psi_rev);
    BitReverseVector(psi_inv_rev);
    for (int j = 0; j < degree; j++) {
      psi_rev[j] = primeutil::ToMontgomery<uint32_t>(psi_rev[j], p);
      psi_inv_rev[j] = primeutil::ToMontgomery<uint32_t>(psi_inv_rev[j], p);
    }
    int32_t norm_hi = basic::Normalize<uint32_t>(p - 1, p);
    int32_t norm_mid = basic::Normalize<uint32_t>(p >> 1, p);
    uint32_t pw = primeutil::PowMod<uint32_t>(12345, -77, p);
    std::printf(
        "{\"prime\": %u, \"generator\": %u, \"psi\": %u, \"psi_inv\": %u, "
        "\"q_inv\": %d, \"n_inv\": %u, \"r2\": %u, \"tw_hash\": \"%016llx\", "
        "\"itw_hash\": \"%016llx\", \"tw_head\": [%u, %u, %u, %u], "
        "\"normalize_hi\": %d, \"normalize_mid\": %d, \"pow_neg\": %u}\n",
        p, g, psi, psi_inv, qinv, n_inv, r2, fnv(psi_rev), fnv(psi_inv_rev),
        psi_rev[0], psi_rev[1], psi_rev[2], psi_rev[3], norm_hi, norm_mid, pw);
  }
  return 0;
}
