"""The header-only C++ mirror (include/cheddar_b200.hpp), including its
bootstrapping classes, compiles and links
against the C ABI library, and reports a parameter error by exception (no
GPU needed: the JSON is rejected before any device call)."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include "cheddar_b200.hpp"
#include <cstdio>
// compiled, not run: the bootstrapping-side classes of the shim
void unused_paths(cheddar_b200::Context &ctx, const cheddar_b200::EvaluationKey &k) {
  cheddar_b200::EvkMap m(ctx);
  m.SetMultiplicationKey(k);
  m.SetConjugationKey(k);
  m.AddRotationKey(1, k);
  cheddar_b200::BootContext bc(ctx, 1 << 15);
  cheddar_b200::BootContext bc_sparse(ctx, 1 << 12, 4, 3, 5, CHD_BOOT_IMAGINARY_REMOVING);
  std::vector<int> r = bc.RequiredRotations();
  cheddar_b200::Ciphertext a(ctx), b(ctx);
  bc.ModUpToMax(b, a, m);
  m.SetDenseToSparseKey(k);
  m.SetSparseToDenseKey(k);
  bc.Boot(b, a, m);
  bc.BootBatch({&b}, {&a}, m);
  std::vector<uint32_t> cx = ctx.EncodeConstant(0, 1.0, 0.5);
  ctx.SetKeySwitchEngine(CHD_BCONV_TENSOR_CORE);
  ctx.Copy(b, a);
  ctx.MultUnsafe(b, a, a, 3);
  ctx.MultUnsafe(b, a, cx, 0, 1.0);
  ctx.MadUnsafe(b, a, cx, 0, 1.0);
  ctx.Permute(b, a, 3);
  ctx.PermuteConjugate(b, a);
  ctx.HConjAdd(b, a, a, k);
  ctx.LevelDown(b, a, 0);
  ctx.MultKeyNoModDown(b, a, k);
  const uint32_t *pt = nullptr;
  ctx.Add(b, a, pt, 1.0);
  ctx.Sub(b, a, pt, 1.0);
  ctx.Sub(b, pt, 1.0, a);
  ctx.Mult(b, a, pt, 1.0);
  ctx.MultUnsafe(b, a, pt, 3, 0, 1.0, -1);
  ctx.Add(b, a, cx);
  ctx.Mult(b, a, cx, 1.0);
  ctx.Sub(b, a, cx);
  ctx.Sub(b, cx, 1.0, a);
  bool compat = ctx.IsMultUnsafeCompatible(1, 2);
  (void)compat;
  int eng = ctx.KeySwitchEngine();
  ctx.HMultBatch({&b}, {&a}, {&a}, k, true);
  ctx.BeginGraph();
  chd_graph *g = ctx.EndGraph();
  ctx.LaunchGraph(g);
  chd_graph_destroy(g);
  (void)r;
  (void)cx;
  (void)eng;
}
int main() {
  try {
    auto ctx = cheddar_b200::Context::Create("{\"log_degree\": 16}");
    (void)ctx;
    return 2;
  } catch (const cheddar_b200::Error &e) {
    std::printf("%d %s\n", e.code, e.what());
    return e.code == CHD_ERR_PARSE ? 0 : 3;
  }
}
'''


def test_cpp_shim_compiles_and_reports_errors():
    lib_dir = os.path.join(ROOT, "cheddar-fhe_b200")
    if not os.path.exists(os.path.join(lib_dir, "libcheddar_b200.so")):
        pytest.skip("library not built")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        open(src, "w").write(SRC)
        subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
                        "-L", lib_dir, "-lcheddar_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
        out = subprocess.run([exe], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "Missing" in out.stdout
