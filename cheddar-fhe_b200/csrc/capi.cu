// C ABI over the host evaluator (include/cheddar_b200.h).
#include <cstring>

#include <algorithm>
#include <exception>
#include <complex>

#include "../../include/cheddar_b200.h"
#include "host.h"

using namespace chd;

struct chd_evk_map {
  RotKeys rot;
  const DeviceEvk *conj = nullptr, *mult = nullptr, *dts = nullptr, *std_key = nullptr;
  ProgKeys keys() const {
    ProgKeys k;
    k.mult = mult;
    k.conj = conj;
    k.dts = dts;
    k.std_key = std_key;
    k.rot = &rot;
    return k;
  }
};
struct chd_lintrans {
  LTPlan plan;
};
struct chd_boot {
  BootPlan plan;
  std::vector<DeviceCt> regs;  // program registers kept across calls
  std::vector<std::vector<DeviceCt>> batch_regs;  // per batch member, chd_boot_run_batch
};
struct chd_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~chd_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};
struct chd_program {
  Program prog;
  double start_scale = 0, end_scale = 0;
  int out_level = 0;
};

namespace {
int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}
#define CHD_NOTNULL(p) \
  if (!(p)) return fail(CHD_ERR_INVALID_ARG, std::string(__func__) + ": null argument " #p)
// a non-null context, made current (its device) for the rest of the call
#define CHD_CTX(ctx) \
  CHD_NOTNULL(ctx);  \
  DeviceGuard device_guard_(ctx->c->device)
// the kernels move device data in 16-byte vectors
#define CHD_ALIGNED(p)                                    \
  if (reinterpret_cast<uintptr_t>(p) & 15)                \
  return fail(CHD_ERR_INVALID_ARG, std::string(__func__) + ": device pointer " #p " is not 16-byte aligned")
}  // namespace

extern "C" {

const char *chd_last_error(void) { return last_error(); }

int chd_context_create_json(const char *json_text, int device, chd_context **out) try {
  CHD_NOTNULL(json_text);
  CHD_NOTNULL(out);
  ParamSpec spec;
  std::string err;
  if (!parse_param_json(json_text, &spec, &err)) return fail(CHD_ERR_PARSE, err);
  auto c = Context::create(spec, device, &err);
  if (!c) return fail(CHD_ERR_INVALID_ARG, err);
  *out = new chd_context{std::move(c)};
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_context_create(int log_degree, double base_scale, int default_encryption_level, const int *level_config,
                       int num_levels, const uint32_t *main_primes, int num_main, const uint32_t *aux_primes,
                       int num_aux, const uint32_t *ter_primes, int num_ter, int additional_main,
                       int additional_ter, int device, chd_context **out) try {
  CHD_NOTNULL(level_config);
  CHD_NOTNULL(main_primes);
  CHD_NOTNULL(aux_primes);
  CHD_NOTNULL(out);
  if (num_ter > 0 && !ter_primes) return fail(CHD_ERR_INVALID_ARG, "ter_primes is null");
  ParamSpec s;
  s.log_degree = log_degree;
  s.base_scale = base_scale;
  s.default_encryption_level = default_encryption_level;
  for (int i = 0; i < num_levels; i++) s.level_config.emplace_back(level_config[2 * i], level_config[2 * i + 1]);
  s.main_primes.assign(main_primes, main_primes + num_main);
  s.aux_primes.assign(aux_primes, aux_primes + num_aux);
  if (num_ter > 0) s.ter_primes.assign(ter_primes, ter_primes + num_ter);
  s.additional_base = {additional_main, additional_ter};
  std::string err;
  auto c = Context::create(s, device, &err);
  if (!c) return fail(CHD_ERR_INVALID_ARG, err);
  *out = new chd_context{std::move(c)};
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_context_destroy(chd_context *ctx) {
  if (!ctx) return;
  DeviceGuard device_guard(ctx->c->device);
  delete ctx;
}

int chd_context_set_stream(chd_context *ctx, void *cuda_stream) try {
  CHD_CTX(ctx);
  Context &C = *ctx->c;
  if (C.own_stream && C.stream) {
    cudaStreamSynchronize(C.stream);
  }
  if (cuda_stream) {
    if (C.own_stream && C.stream) cudaStreamDestroy(C.stream);
    C.own_stream = false;
    C.stream = static_cast<cudaStream_t>(cuda_stream);
  } else if (!C.own_stream) {
    cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking);
    C.own_stream = true;
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_stage_timing(chd_context *ctx, int enable) try {
  CHD_CTX(ctx);
  Context &C = *ctx->c;
  if (enable) {
    C.timer.used = 0;
    C.timer.spans.clear();
  }
  C.timer.on = enable != 0;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_copy(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->copy_ct(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_unsafe(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
                    int level) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(b);
  return ctx->c->mult_unsafe(res->ct, a->ct, b->ct, level);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_unsafe_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx,
                          int const_level, double const_scale, int level) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(cx);
  return ctx->c->mult_unsafe_const(res->ct, a->ct, cx, const_level, const_scale, level);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mad_unsafe(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx,
                   int const_level, double const_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(cx);
  return ctx->c->mad_unsafe(res->ct, a->ct, cx, const_level, const_scale);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_permute(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, int rot_dist) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->permute_ct(res->ct, a->ct, rot_dist, false);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_permute_conjugate(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->permute_ct(res->ct, a->ct, 0, true);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hconj_add(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
                  const chd_evk *conj_key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(b);
  CHD_NOTNULL(conj_key);
  return ctx->c->hconj_add(res->ct, a->ct, b->ct, conj_key->k);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_level_down(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, int target_level) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->level_down(res->ct, a->ct, target_level);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_key_no_moddown(chd_context *ctx, chd_ciphertext *accum, const chd_ciphertext *a, const chd_evk *key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(accum);
  CHD_NOTNULL(a);
  CHD_NOTNULL(key);
  return ctx->c->mult_key_no_moddown(accum->ct, a->ct, key->k);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_unsafe_compatible(const chd_context *ctx, int level1, int level2) try {
  if (!ctx) return -1;
  const int ml = ctx->c->P->max_level;
  if (level1 < 0 || level2 < 0 || level1 > ml || level2 > ml) return -1;
  return ctx->c->mult_unsafe_compatible(level1, level2) ? 1 : 0;
} catch (const std::exception &e) {
  fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
  return -1;
} catch (...) {
  fail(CHD_ERR_INTERNAL, "internal error");
  return -1;
}

int chd_add_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                  double pt_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  return ctx->c->add_sub_plain(res->ct, a->ct, pt_dev, pt_scale, false);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_sub_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                  double pt_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  return ctx->c->add_sub_plain(res->ct, a->ct, pt_dev, pt_scale, true);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_sub_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(cx);
  return ctx->c->sub_const(res->ct, a->ct, cx);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_sub_plain_ct(chd_context *ctx, chd_ciphertext *res, const uint32_t *pt_dev, double pt_scale,
                     const chd_ciphertext *b) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  CHD_NOTNULL(b);
  return ctx->c->sub_from(res->ct, pt_dev, nullptr, pt_scale, b->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_sub_const_ct(chd_context *ctx, chd_ciphertext *res, const uint32_t *cx, double const_scale,
                     const chd_ciphertext *b) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(cx);
  CHD_NOTNULL(b);
  return ctx->c->sub_from(res->ct, nullptr, cx, const_scale, b->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_unsafe_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                          int pt_level, int pt_num_aux, double pt_scale, int level) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  return ctx->c->mult_unsafe_plain(res->ct, a->ct, pt_dev, pt_level, pt_num_aux, pt_scale, level);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_set_ks_engine(chd_context *ctx, int engine) try {
  CHD_CTX(ctx);
  if (engine != CHD_BCONV_CUDA_CORE && engine != CHD_BCONV_TENSOR_CORE && engine != CHD_BCONV_AUTO &&
      engine != CHD_BCONV_TENSOR_CORE_WIDE)
    return fail(CHD_ERR_INVALID_ARG,
                "chd_set_ks_engine: engine must be CHD_BCONV_CUDA_CORE, CHD_BCONV_TENSOR_CORE, "
                "CHD_BCONV_TENSOR_CORE_WIDE or CHD_BCONV_AUTO");
  ctx->c->ks_engine = engine;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_get_ks_engine(const chd_context *ctx) { return ctx ? ctx->c->ks_engine : -1; }

int chd_ks_tuned_shapes(int *out, int cap) { return modswitch_tuned_shapes(out, cap); }

int chd_ks_rows_tuned_shapes(int *out, int cap) { return ks_rows_tuned_shapes(out, cap); }

int chd_set_stream_split(chd_context *ctx, int on) try {
  CHD_CTX(ctx);
  ctx->c->split_streams = on != 0;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_get_stream_split(const chd_context *ctx) { return ctx ? (ctx->c->split_streams ? 1 : 0) : -1; }

int chd_stage_times(chd_context *ctx, double *ms, int *launches) try {
  CHD_CTX(ctx);
  if (!ms || !launches) return fail(CHD_ERR_INVALID_ARG, "chd_stage_times: null output");
  return ctx->c->timer_read(ms, launches);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_context_synchronize(chd_context *ctx) try {
  CHD_CTX(ctx);
  Context &C = *ctx->c;
  cudaError_t e = cudaStreamSynchronize(C.stream);
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  // a kernel whose bounded wait ran out leaves 1 in the device error word
  int flag = 0;
  e = cudaMemcpy(&flag, C.d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  if (flag) {
    cudaMemset(C.d_err, 0, sizeof(int));
    return fail(CHD_ERR_CUDA, "a kernel gave up waiting for its tensor-core work (bounded wait ran out)");
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_debug_stall_tensor_waits(chd_context *ctx, int polls) try {
  CHD_CTX(ctx);
  if (polls < 0) return fail(CHD_ERR_INVALID_ARG, "chd_debug_stall_tensor_waits: polls must be >= 0");
  ctx->c->tc_stall_polls = static_cast<uint32_t>(polls);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_level_np(const chd_context *ctx, int level, int *num_main, int *num_ter) try {
  CHD_CTX(ctx);
  const Params &P = *ctx->c->P;
  if (level < -1 || level > P.max_level) return fail(CHD_ERR_INVALID_LEVEL, "invalid level");
  NP np = P.level_np(level, 0);
  if (num_main) *num_main = np.main;
  if (num_ter) *num_ter = np.ter;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}
int chd_max_level(const chd_context *ctx) { return ctx ? ctx->c->P->max_level : -1; }
int chd_degree(const chd_context *ctx) { return ctx ? ctx->c->P->n : -1; }
int chd_alpha(const chd_context *ctx) { return ctx ? ctx->c->P->alpha : -1; }
int chd_num_q_primes(const chd_context *ctx) { return ctx ? ctx->c->P->L : -1; }
double chd_scale(const chd_context *ctx, int level) {
  if (!ctx) return 0.0;
  const Params &P = *ctx->c->P;
  if (level == -1) level = 0;
  if (level < 0 || level >= static_cast<int>(P.scale.size())) return 0.0;
  return P.scale[level];
}
double chd_rescale_prime_prod(const chd_context *ctx, int level) {
  if (!ctx) return 0.0;
  const Params &P = *ctx->c->P;
  if (level < 1 || level > P.max_level) return 0.0;
  return P.rescale_prod[level];
}
int chd_prime_gidx(const chd_context *ctx, int num_main, int num_ter, int num_aux, int *out) try {
  if (!ctx || !out) return -1;
  NP np{num_main, num_ter, num_aux};
  ctx->c->P->gidx(np, out);
  return np.total();
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ct_create(chd_context *ctx, chd_ciphertext **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(out);
  *out = new chd_ciphertext();
  (*out)->ct.num_slots = ctx->c->P->n / 2;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_ct_destroy(chd_ciphertext *ct) { delete ct; }

int chd_ct_wrap(chd_context *ctx, int num_main, int num_ter, int num_aux, int has_rx, double scale, int num_slots,
                uint32_t *bx, uint32_t *ax, uint32_t *rx, size_t words_per_part, chd_ciphertext **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(out);
  CHD_NOTNULL(bx);
  CHD_NOTNULL(ax);
  if (has_rx && !rx) return fail(CHD_ERR_INVALID_ARG, "chd_ct_wrap: rx is null");
  CHD_ALIGNED(bx);
  CHD_ALIGNED(ax);
  CHD_ALIGNED(has_rx ? rx : nullptr);
  NP np{num_main, num_ter, num_aux};
  if (static_cast<size_t>(np.total()) * ctx->c->P->n > words_per_part)
    return fail(CHD_ERR_SHAPE, "chd_ct_wrap: buffers smaller than the ciphertext");
  auto *c = new chd_ciphertext();
  c->ct.owned = false;
  c->ct.np = np;
  c->ct.has_rx = has_rx != 0;
  c->ct.scale = scale;
  c->ct.num_slots = num_slots;
  c->ct.bx = bx;
  c->ct.ax = ax;
  c->ct.rx = has_rx ? rx : nullptr;
  c->ct.cap_words = words_per_part;
  *out = c;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ct_import(chd_context *ctx, chd_ciphertext *ct, int num_main, int num_ter, int num_aux, int has_rx,
                  double scale, int num_slots, const uint32_t *bx, const uint32_t *ax, const uint32_t *rx,
                  int src_on_device) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(ct);
  CHD_NOTNULL(bx);
  CHD_NOTNULL(ax);
  if (has_rx && !rx) return fail(CHD_ERR_INVALID_ARG, "chd_ct_import: rx is null");
  Context &C = *ctx->c;
  NP np{num_main, num_ter, num_aux};
  if (C.P->np_to_level(NP{num_main, num_ter, 0}) < -1 || num_aux < 0 || num_aux > C.P->alpha)
    return fail(CHD_ERR_INVALID_LEVEL, "chd_ct_import: (num_main, num_ter) is not a level");
  int rc = ct->ct.reserve(np, has_rx != 0, C.P->n);
  if (rc) return rc;
  const size_t bytes = static_cast<size_t>(np.total()) * C.P->n * 4;
  cudaMemcpyKind kind = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(ct->ct.bx, bx, bytes, kind, C.stream);
  cudaMemcpyAsync(ct->ct.ax, ax, bytes, kind, C.stream);
  if (has_rx) cudaMemcpyAsync(ct->ct.rx, rx, bytes, kind, C.stream);
  ct->ct.scale = scale;
  ct->ct.num_slots = num_slots;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  if (!src_on_device) cudaStreamSynchronize(C.stream);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ct_export(chd_context *ctx, const chd_ciphertext *ct, uint32_t *bx, uint32_t *ax, uint32_t *rx,
                  int dst_on_device) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(ct);
  Context &C = *ctx->c;
  const size_t bytes = static_cast<size_t>(ct->ct.np.total()) * C.P->n * 4;
  cudaMemcpyKind kind = dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (bx) cudaMemcpyAsync(bx, ct->ct.bx, bytes, kind, C.stream);
  if (ax) cudaMemcpyAsync(ax, ct->ct.ax, bytes, kind, C.stream);
  if (rx && ct->ct.has_rx) cudaMemcpyAsync(rx, ct->ct.rx, bytes, kind, C.stream);
  cudaError_t e = cudaStreamSynchronize(C.stream);
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ct_info(const chd_ciphertext *ct, int *num_main, int *num_ter, int *num_aux, int *has_rx, double *scale,
                int *num_slots) try {
  CHD_NOTNULL(ct);
  if (num_main) *num_main = ct->ct.np.main;
  if (num_ter) *num_ter = ct->ct.np.ter;
  if (num_aux) *num_aux = ct->ct.np.aux;
  if (has_rx) *has_rx = ct->ct.has_rx;
  if (scale) *scale = ct->ct.scale;
  if (num_slots) *num_slots = ct->ct.num_slots;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ct_device_ptrs(const chd_ciphertext *ct, uint32_t **bx, uint32_t **ax, uint32_t **rx) try {
  CHD_NOTNULL(ct);
  if (bx) *bx = ct->ct.bx;
  if (ax) *ax = ct->ct.ax;
  if (rx) *rx = ct->ct.rx;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_create(chd_context *ctx, int beta, const uint32_t *bx, const uint32_t *ax, int src_on_device,
                   chd_evk **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(bx);
  CHD_NOTNULL(ax);
  CHD_NOTNULL(out);
  Context &C = *ctx->c;
  const int need = (C.P->L + C.P->alpha - 1) / C.P->alpha;
  if (beta < need || beta > 8) return fail(CHD_ERR_KEY, "chd_evk_create: beta must cover all q primes (<= 8)");
  auto *k = new chd_evk();
  k->k.beta = beta;
  k->k.np = NP{C.P->max_main, C.P->max_ter, C.P->alpha};
  const size_t bytes = static_cast<size_t>(beta) * (C.P->L + C.P->alpha) * C.P->n * 4;
  if (cudaMalloc(&k->k.bx, bytes) != cudaSuccess || cudaMalloc(&k->k.ax, bytes) != cudaSuccess) {
    delete k;
    return fail(CHD_ERR_ALLOC, "chd_evk_create: device allocation failed");
  }
  cudaMemcpyKind kind = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(k->k.bx, bx, bytes, kind, C.stream);
  cudaMemcpyAsync(k->k.ax, ax, bytes, kind, C.stream);
  cudaError_t e = cudaStreamSynchronize(C.stream);
  if (e != cudaSuccess) {
    delete k;
    return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_evk_destroy(chd_evk *evk) { delete evk; }

int chd_evk_info(const chd_evk *evk, int *beta, int *num_main, int *num_ter, int *num_aux) try {
  CHD_NOTNULL(evk);
  if (beta) *beta = evk->k.beta;
  if (num_main) *num_main = evk->k.np.main;
  if (num_ter) *num_ter = evk->k.np.ter;
  if (num_aux) *num_aux = evk->k.np.aux;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_export(chd_context *ctx, const chd_evk *evk, uint32_t *bx, uint32_t *ax, int dst_on_device) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(evk);
  CHD_NOTNULL(bx);
  CHD_NOTNULL(ax);
  const size_t bytes = static_cast<size_t>(evk->k.beta) * evk->k.np.total() * ctx->c->P->n * 4;
  const cudaMemcpyKind kind = dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  Context &C = *ctx->c;
  cudaMemcpyAsync(bx, evk->k.bx, bytes, kind, C.stream);
  cudaMemcpyAsync(ax, evk->k.ax, bytes, kind, C.stream);
  const cudaError_t e = cudaStreamSynchronize(C.stream);
  return e == cudaSuccess ? CHD_OK : fail(CHD_ERR_CUDA, cudaGetErrorString(e));
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

#define CTX_CT3(name, call)                                                                              \
  int name(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b) { \
    CHD_CTX(ctx);                                                                                  \
    CHD_NOTNULL(res);                                                                                  \
    CHD_NOTNULL(a);                                                                                    \
    CHD_NOTNULL(b);                                                                                    \
    return ctx->c->call(res->ct, a->ct, b->ct);                                                        \
  }
CTX_CT3(chd_add, add)
CTX_CT3(chd_sub, sub)
CTX_CT3(chd_mult, mult_tensor)
#undef CTX_CT3

int chd_neg(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->neg(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx,
                   double const_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(cx);
  return ctx->c->mult_const(res->ct, a->ct, cx, const_scale);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_add_const(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *cx) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(cx);
  return ctx->c->add_const(res->ct, a->ct, cx);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_plain(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const uint32_t *pt_dev,
                   double pt_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  return ctx->c->mult_plain(res->ct, a->ct, pt_dev, pt_scale);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_imaginary_unit(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->mult_imag_unit(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_rescale(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->rescale(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_encode(chd_context *ctx, int level, double scale, const double *re, const double *im, int msg_len,
               int num_aux, uint32_t *pt_dev, int *num_slots) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(re);
  CHD_NOTNULL(im);
  CHD_NOTNULL(pt_dev);
  CHD_ALIGNED(pt_dev);
  if (msg_len < 1) return fail(CHD_ERR_INVALID_ARG, "chd_encode: empty message");
  std::vector<std::complex<double>> msg(msg_len);
  for (int i = 0; i < msg_len; i++) msg[i] = std::complex<double>(re[i], im[i]);
  return ctx->c->encode(level, scale, msg.data(), msg_len, num_aux, pt_dev, num_slots);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_decode(chd_context *ctx, int level, double scale, const uint32_t *pt_dev, int num_slots, double *re,
               double *im) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(pt_dev);
  CHD_NOTNULL(re);
  CHD_NOTNULL(im);
  CHD_ALIGNED(pt_dev);
  std::vector<std::complex<double>> out(num_slots > 0 ? num_slots : 1);
  int rc = ctx->c->decode(level, scale, pt_dev, num_slots, out.data());
  if (rc != CHD_OK) return rc;
  for (int i = 0; i < num_slots; i++) {
    re[i] = out[i].real();
    im[i] = out[i].imag();
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_encode_const(chd_context *ctx, int level, double scale, double value, int num_aux, uint32_t *cx) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(cx);
  const Params &P = *ctx->c->P;
  if (level < -1 || level > P.max_level) return fail(CHD_ERR_INVALID_LEVEL, "chd_encode_const: invalid level");
  if (num_aux < 0 || num_aux > P.alpha) return fail(CHD_ERR_INVALID_ARG, "chd_encode_const: invalid aux count");
  std::vector<uint32_t> v;
  ctx->c->encode_const(level, scale, value, num_aux, &v);
  std::copy(v.begin(), v.end(), cx);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_modup_to_max(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk_map *keys) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  Context &C = *ctx->c;
  if (C.uses_sse()) {
    if (!keys || !keys->dts || !keys->std_key)
      return fail(CHD_ERR_KEY, "chd_modup_to_max: dense-to-sparse and sparse-to-dense keys required");
    if (res == a) {
      DeviceCt tmp;
      int rc = C.modup_to_max_sse(tmp, a->ct, *keys->dts, *keys->std_key);
      if (rc != CHD_OK) return rc;
      swap_regs(res->ct, tmp);
      return CHD_OK;
    }
    return C.modup_to_max_sse(res->ct, a->ct, *keys->dts, *keys->std_key);
  }
  return C.modup_to_max(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_map_create(chd_context *ctx, chd_evk_map **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(out);
  *out = new chd_evk_map();
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_evk_map_destroy(chd_evk_map *m) { delete m; }

int chd_evk_map_set_rotation(chd_evk_map *m, int rot_idx, const chd_evk *key) try {
  CHD_NOTNULL(m);
  CHD_NOTNULL(key);
  if (rot_idx <= 0) return fail(CHD_ERR_INVALID_ARG, "chd_evk_map_set_rotation: rotation index must be positive");
  m->rot[rot_idx] = &key->k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_map_set_conjugation(chd_evk_map *m, const chd_evk *key) try {
  CHD_NOTNULL(m);
  CHD_NOTNULL(key);
  m->conj = &key->k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_map_set_mult(chd_evk_map *m, const chd_evk *key) try {
  CHD_NOTNULL(m);
  CHD_NOTNULL(key);
  m->mult = &key->k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_map_set_dense_to_sparse(chd_evk_map *m, const chd_evk *key) try {
  CHD_NOTNULL(m);
  CHD_NOTNULL(key);
  m->dts = &key->k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_map_set_sparse_to_dense(chd_evk_map *m, const chd_evk *key) try {
  CHD_NOTNULL(m);
  CHD_NOTNULL(key);
  m->std_key = &key->k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evk_create_np(chd_context *ctx, int num_main, int num_ter, int num_aux, int beta, const uint32_t *bx,
                      const uint32_t *ax, int src_on_device, chd_evk **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(bx);
  CHD_NOTNULL(ax);
  CHD_NOTNULL(out);
  Context &C = *ctx->c;
  if (num_main < 0 || num_ter < 0 || num_aux < 1 || num_main > C.P->max_main || num_ter > C.P->max_ter ||
      num_aux > C.P->alpha || beta < 1 || beta > 8)
    return fail(CHD_ERR_KEY, "chd_evk_create_np: invalid key basis");
  auto *k = new chd_evk();
  k->k.beta = beta;
  k->k.np = NP{num_main, num_ter, num_aux};
  const size_t bytes = static_cast<size_t>(beta) * (num_main + num_ter + num_aux) * C.P->n * 4;
  if (cudaMalloc(&k->k.bx, bytes) != cudaSuccess || cudaMalloc(&k->k.ax, bytes) != cudaSuccess) {
    delete k;
    return fail(CHD_ERR_ALLOC, "chd_evk_create_np: device allocation failed");
  }
  cudaMemcpyKind kind = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(k->k.bx, bx, bytes, kind, C.stream);
  cudaMemcpyAsync(k->k.ax, ax, bytes, kind, C.stream);
  cudaError_t e = cudaStreamSynchronize(C.stream);
  if (e != cudaSuccess) {
    delete k;
    return fail(CHD_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = k;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_lintrans_create(chd_context *ctx, int width, int n_diag, const int *diag_idx, const double *re,
                        const double *im, int pt_level, double pt_scale, int bs, int gs, int pre_rotation,
                        int additional_pt_rot, chd_lintrans **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(diag_idx);
  CHD_NOTNULL(re);
  CHD_NOTNULL(im);
  CHD_NOTNULL(out);
  if (width <= 0 || n_diag <= 0 || bs <= 0 || gs <= 0) return fail(CHD_ERR_INVALID_ARG, "chd_lintrans_create: bad shape");
  SMat m;
  m.h = m.w = width;
  for (int i = 0; i < n_diag; i++) {
    if (diag_idx[i] < 0 || diag_idx[i] >= width) return fail(CHD_ERR_INVALID_ARG, "chd_lintrans_create: bad diagonal");
    std::vector<std::complex<double>> v(width);
    for (int k = 0; k < width; k++)
      v[k] = std::complex<double>(re[static_cast<size_t>(i) * width + k], im[static_cast<size_t>(i) * width + k]);
    m.d[diag_idx[i]] = std::move(v);
  }
  auto *lt = new chd_lintrans();
  int rc = ctx->c->lt_build(m, pt_level, pt_scale, bs, gs, pre_rotation, additional_pt_rot, false, &lt->plan);
  if (rc != CHD_OK) {
    delete lt;
    return rc;
  }
  *out = lt;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_lintrans_destroy(chd_lintrans *lt) { delete lt; }

namespace {
// HoistHandler::AddRequiredRotations (Hoist.cu:977-1003)
int plan_rotations(const LTPlan &p, bool min_ks, std::vector<int> *r) {
  if (min_ks) {
    int bs = 0, gs = 0;
    const int rc = lt_min_ks_strides(p, &bs, &gs);
    if (rc != CHD_OK) return rc;
    if (bs) r->push_back(bs);
    if (gs) r->push_back(gs);
    return CHD_OK;
  }
  for (int b : p.bs_idx)
    if (b) r->push_back(b);
  for (int g : p.gs_idx)
    if (g) r->push_back(g);
  return CHD_OK;
}
}  // namespace

int chd_lintrans_rotations(const chd_lintrans *lt, int min_ks, int *out, int cap, int *count) try {
  CHD_NOTNULL(lt);
  CHD_NOTNULL(count);
  std::vector<int> r;
  int rc = plan_rotations(lt->plan, min_ks != 0, &r);
  if (rc != CHD_OK) return rc;
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
  *count = static_cast<int>(r.size());
  if (out)
    for (int i = 0; i < std::min(cap, *count); i++) out[i] = r[i];
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_lintrans_num_pts(const chd_lintrans *lt, int *count) try {
  CHD_NOTNULL(lt);
  CHD_NOTNULL(count);
  *count = static_cast<int>(lt->plan.pts.size());
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_lintrans_pt(const chd_lintrans *lt, int i, int *gs, int *bs, double *re, double *im) try {
  CHD_NOTNULL(lt);
  if (i < 0 || i >= static_cast<int>(lt->plan.pts.size())) return fail(CHD_ERR_INVALID_ARG, "chd_lintrans_pt: index");
  const LTPlan::Pt &p = lt->plan.pts[i];
  if (gs) *gs = p.gs;
  if (bs) *bs = p.bs;
  for (size_t k = 0; k < p.msg.size(); k++) {
    if (re) re[k] = p.msg[k].real();
    if (im) im[k] = p.msg[k].imag();
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_lintrans_evaluate(chd_context *ctx, const chd_lintrans *lt, chd_ciphertext *res, const chd_ciphertext *in,
                          const chd_evk_map *keys, int min_ks) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(lt);
  CHD_NOTNULL(res);
  CHD_NOTNULL(in);
  CHD_NOTNULL(keys);
  if (min_ks) {
    if (res == in) {
      DeviceCt tmp;
      int rc = ctx->c->lt_evaluate_min_ks(tmp, in->ct, lt->plan, keys->rot);
      if (rc != CHD_OK) return rc;
      swap_regs(res->ct, tmp);
      return CHD_OK;
    }
    return ctx->c->lt_evaluate_min_ks(res->ct, in->ct, lt->plan, keys->rot);
  }
  if (res == in) {
    DeviceCt tmp;
    int rc = ctx->c->lt_evaluate(tmp, in->ct, lt->plan, keys->rot);
    if (rc != CHD_OK) return rc;
    std::swap(res->ct.bx, tmp.bx);
    std::swap(res->ct.ax, tmp.ax);
    std::swap(res->ct.rx, tmp.rx);
    std::swap(res->ct.cap_words, tmp.cap_words);
    std::swap(res->ct.owned, tmp.owned);
    res->ct.np = tmp.np;
    res->ct.has_rx = tmp.has_rx;
    res->ct.scale = tmp.scale;
    res->ct.num_slots = tmp.num_slots;
    return CHD_OK;
  }
  return ctx->c->lt_evaluate(res->ct, in->ct, lt->plan, keys->rot);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_poly_create(chd_context *ctx, const double *coeffs, int n, int input_level, double input_scale,
                    double target_scale, int chebyshev, chd_program **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(coeffs);
  CHD_NOTNULL(out);
  if (n < 1) return fail(CHD_ERR_INVALID_ARG, "chd_poly_create: no coefficients");
  auto *pg = new chd_program();
  pg->prog.input = pg->prog.reg();
  int reg = -1;
  int rc = ctx->c->compile_poly(pg->prog, pg->prog.input, std::vector<double>(coeffs, coeffs + n), input_level,
                                input_scale, target_scale, chebyshev != 0, &reg, &pg->out_level);
  if (rc != CHD_OK) {
    delete pg;
    return rc;
  }
  pg->prog.output = reg;
  pg->start_scale = input_scale;
  pg->end_scale = target_scale;
  *out = pg;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_evalmod_create(chd_context *ctx, int start_level, const double *coeffs, int n, int num_double_angle,
                       int initial_K, chd_program **out, double *start_scale, double *end_scale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(coeffs);
  CHD_NOTNULL(out);
  auto *pg = new chd_program();
  pg->prog.input = pg->prog.reg();
  int reg = -1;
  int rc = ctx->c->compile_evalmod(pg->prog, pg->prog.input, start_level, std::vector<double>(coeffs, coeffs + n),
                                   num_double_angle, initial_K, &reg, &pg->out_level, &pg->start_scale,
                                   &pg->end_scale);
  if (rc != CHD_OK) {
    delete pg;
    return rc;
  }
  pg->prog.output = reg;
  if (start_scale) *start_scale = pg->start_scale;
  if (end_scale) *end_scale = pg->end_scale;
  *out = pg;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_program_destroy(chd_program *p) { delete p; }

int chd_boot_mod_coefficients(double *out, int cap) try {
  const auto &c = boot_mod_coefficients();
  if (out)
    for (int i = 0; i < std::min(cap, static_cast<int>(c.size())); i++) out[i] = c[i];
  return static_cast<int>(c.size());
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_program_json(const chd_program *p, char *buf, size_t cap, size_t *len) try {
  CHD_NOTNULL(p);
  CHD_NOTNULL(len);
  const Program &g = p->prog;
  std::string s;
  char tmp[512];
  snprintf(tmp, sizeof tmp, "{\"nregs\":%d,\"input\":%d,\"output\":%d,\"out_level\":%d,\"consts\":[", g.nregs,
           g.input, g.output, p->out_level);
  s += tmp;
  for (size_t i = 0; i < g.consts.size(); i++) {
    snprintf(tmp, sizeof tmp, "%s[%d,%.17g,%.17g]", i ? "," : "", g.consts[i].level, g.consts[i].scale,
             g.consts[i].value);
    s += tmp;
  }
  s += "],\"ops\":[";
  for (size_t i = 0; i < g.ops.size(); i++) {
    const ProgOp &o = g.ops[i];
    snprintf(tmp, sizeof tmp, "%s{\"k\":%d,\"d\":%d,\"a\":%d,\"b\":%d,\"l\":%d,\"c\":%d,\"p\":%d,\"r\":%d,\"sc\":%.17g,\"s\":[",
             i ? "," : "", static_cast<int>(o.kind), o.dst, o.a, o.b, o.level, o.c, o.plain, o.rot, o.scale);
    s += tmp;
    for (size_t j = 0; j < o.srcs.size(); j++) s += (j ? "," : "") + std::to_string(o.srcs[j]);
    s += "],\"cs\":[";
    for (size_t j = 0; j < o.cs.size(); j++) s += (j ? "," : "") + std::to_string(o.cs[j]);
    s += "]}";
  }
  s += "]}";
  *len = s.size() + 1;
  if (buf && cap >= s.size() + 1) memcpy(buf, s.c_str(), s.size() + 1);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

namespace {
Status copy_ct(Context &C, DeviceCt &dst, const DeviceCt &src) {
  CHD_TRY(dst.reserve(src.np, src.has_rx, C.P->n));
  const size_t bytes = static_cast<size_t>(src.np.total()) * C.P->n * 4;
  cudaMemcpyAsync(dst.bx, src.bx, bytes, cudaMemcpyDeviceToDevice, C.stream);
  cudaMemcpyAsync(dst.ax, src.ax, bytes, cudaMemcpyDeviceToDevice, C.stream);
  if (src.has_rx) cudaMemcpyAsync(dst.rx, src.rx, bytes, cudaMemcpyDeviceToDevice, C.stream);
  dst.scale = src.scale;
  dst.num_slots = src.num_slots;
  return kOk;
}
}  // namespace

int chd_program_run(chd_context *ctx, const chd_program *p, chd_ciphertext *res, const chd_ciphertext *in,
                    const chd_evk_map *keys) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(p);
  CHD_NOTNULL(res);
  CHD_NOTNULL(in);
  Context &C = *ctx->c;
  std::vector<DeviceCt> regs;
  int rc = C.program_regs(p->prog, regs);
  if (rc != CHD_OK) return rc;
  rc = copy_ct(C, regs[p->prog.input], in->ct);
  if (rc != CHD_OK) return rc;
  rc = C.run_program(p->prog, regs, keys ? keys->keys() : ProgKeys{}, nullptr);
  if (rc != CHD_OK) return rc;
  rc = copy_ct(C, res->ct, regs[p->prog.output]);
  if (rc != CHD_OK) return rc;
  return cudaStreamSynchronize(C.stream) == cudaSuccess ? CHD_OK : fail(CHD_ERR_CUDA, "chd_program_run: CUDA error");
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_create(chd_context *ctx, int num_slots, int num_cts_levels, int num_stc_levels, int log_message_ratio,
                    chd_boot **out) try {
  return chd_boot_create_variant(ctx, num_slots, CHD_BOOT_NORMAL, num_cts_levels, num_stc_levels, log_message_ratio,
                                 out);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_create_variant(chd_context *ctx, int num_slots, int variant, int num_cts_levels, int num_stc_levels,
                            int log_message_ratio, chd_boot **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(out);
  auto *b = new chd_boot();
  int rc = ctx->c->boot_build(num_slots, variant, num_cts_levels, num_stc_levels, log_message_ratio, &b->plan);
  if (rc != CHD_OK) {
    delete b;
    return rc;
  }
  *out = b;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_boot_destroy(chd_boot *b) { delete b; }

int chd_boot_rotations(const chd_boot *b, int min_ks, int *out, int cap, int *count) try {
  CHD_NOTNULL(b);
  CHD_NOTNULL(count);
  std::vector<int> r;
  for (const auto &l : b->plan.lts) {
    int rc = plan_rotations(l, min_ks != 0, &r);
    if (rc != CHD_OK) return rc;
  }
  for (int x : b->plan.extra_rotations) r.push_back(x);
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
  *count = static_cast<int>(r.size());
  if (out)
    for (int i = 0; i < std::min(cap, *count); i++) out[i] = r[i];
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_levels(const chd_boot *b, int *levels, double *scales) try {
  CHD_NOTNULL(b);
  const BootPlan &p = b->plan;
  if (levels) {
    levels[0] = p.cts_start;
    levels[1] = p.em_start;
    levels[2] = p.stc_start;
    levels[3] = p.end_level;
    levels[4] = p.log_scaleup;
  }
  if (scales) {
    scales[0] = p.cts_const;
    scales[1] = p.stc_const;
    scales[2] = p.em_start_scale;
    scales[3] = p.em_end_scale;
    scales[4] = p.final_scale;
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_json(const chd_boot *b, char *buf, size_t cap, size_t *len) try {
  CHD_NOTNULL(b);
  chd_program tmp;
  tmp.prog = b->plan.prog;
  tmp.out_level = b->plan.end_level;
  return chd_program_json(&tmp, buf, cap, len);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_lt_info(const chd_boot *b, int i, int *level, double *scale, int *npts, int *width) try {
  CHD_NOTNULL(b);
  if (i < 0 || i >= static_cast<int>(b->plan.lts.size())) return fail(CHD_ERR_INVALID_ARG, "chd_boot_lt_info: index");
  const LTPlan &l = b->plan.lts[i];
  if (level) *level = l.pt_level;
  if (scale) *scale = l.pt_scale;
  if (npts) *npts = static_cast<int>(l.pts.size());
  if (width) *width = l.width;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_lt_pt(const chd_boot *b, int i, int j, int *gs, int *bs, double *re, double *im) try {
  CHD_NOTNULL(b);
  if (i < 0 || i >= static_cast<int>(b->plan.lts.size())) return fail(CHD_ERR_INVALID_ARG, "chd_boot_lt_pt: index");
  const LTPlan &l = b->plan.lts[i];
  if (j < 0 || j >= static_cast<int>(l.pts.size())) return fail(CHD_ERR_INVALID_ARG, "chd_boot_lt_pt: index");
  const LTPlan::Pt &p = l.pts[j];
  if (gs) *gs = p.gs;
  if (bs) *bs = p.bs;
  for (size_t k = 0; k < p.msg.size(); k++) {
    if (re) re[k] = p.msg[k].real();
    if (im) im[k] = p.msg[k].imag();
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_run(chd_context *ctx, chd_boot *b, chd_ciphertext *res, const chd_ciphertext *in, const chd_evk_map *keys,
                 int min_ks) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(b);
  CHD_NOTNULL(res);
  CHD_NOTNULL(in);
  CHD_NOTNULL(keys);
  if (!keys->mult || !keys->conj) return fail(CHD_ERR_KEY, "chd_boot_run: multiplication and conjugation keys required");
  ProgKeys pk = keys->keys();
  pk.min_ks = min_ks != 0;
  if (res == in) {
    DeviceCt tmp;
    int rc = ctx->c->boot_run(b->plan, tmp, in->ct, pk, &b->regs);
    if (rc != CHD_OK) return rc;
    std::swap(res->ct.bx, tmp.bx);
    std::swap(res->ct.ax, tmp.ax);
    std::swap(res->ct.rx, tmp.rx);
    std::swap(res->ct.cap_words, tmp.cap_words);
    std::swap(res->ct.owned, tmp.owned);
    res->ct.np = tmp.np;
    res->ct.has_rx = false;
    res->ct.scale = tmp.scale;
    res->ct.num_slots = tmp.num_slots;
    return CHD_OK;
  }
  return ctx->c->boot_run(b->plan, res->ct, in->ct, pk, &b->regs);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_boot_run_batch(chd_context *ctx, chd_boot *b, int count, chd_ciphertext *const *res,
                       const chd_ciphertext *const *in, const chd_evk_map *keys, int min_ks) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(b);
  CHD_NOTNULL(res);
  CHD_NOTNULL(in);
  CHD_NOTNULL(keys);
  if (count < 1) return fail(CHD_ERR_INVALID_ARG, "chd_boot_run_batch: count must be positive");
  if (!keys->mult || !keys->conj) return fail(CHD_ERR_KEY, "chd_boot_run: multiplication and conjugation keys required");
  for (int c = 0; c < count; c++) {
    if (!res[c] || !in[c]) return fail(CHD_ERR_INVALID_ARG, "chd_boot_run_batch: null ciphertext");
    for (int d = 0; d < count; d++)
      if (d != c && res[c] == res[d]) return fail(CHD_ERR_INVALID_ARG, "chd_boot_run_batch: results must differ");
  }
  ProgKeys pk = keys->keys();
  pk.min_ks = min_ks != 0;
  if (static_cast<int>(b->batch_regs.size()) < count) b->batch_regs.resize(count);
  std::vector<std::vector<DeviceCt> *> regs(count);
  // results written into fresh ciphertexts first when one aliases an input
  std::vector<DeviceCt> tmp(count);
  std::vector<DeviceCt *> out(count);
  std::vector<const DeviceCt *> src(count);
  for (int c = 0; c < count; c++) {
    regs[c] = &b->batch_regs[c];
    src[c] = &in[c]->ct;
    bool alias = false;
    for (int d = 0; d < count; d++) alias = alias || res[c] == in[d];
    out[c] = alias ? &tmp[c] : &res[c]->ct;
  }
  int rc = ctx->c->boot_run_batch(b->plan, count, out.data(), src.data(), pk, regs.data());
  if (rc != CHD_OK) return rc;
  for (int c = 0; c < count; c++) {
    if (out[c] != &tmp[c]) continue;
    DeviceCt &r = res[c]->ct;
    std::swap(r.bx, tmp[c].bx);
    std::swap(r.ax, tmp[c].ax);
    std::swap(r.rx, tmp[c].rx);
    std::swap(r.cap_words, tmp[c].cap_words);
    std::swap(r.owned, tmp[c].owned);
    r.np = tmp[c].np;
    r.has_rx = false;
    r.scale = tmp[c].scale;
    r.num_slots = tmp[c].num_slots;
  }
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_graph_begin(chd_context *ctx) try {
  CHD_CTX(ctx);
  Context &C = *ctx->c;
  if (!C.stream) return fail(CHD_ERR_INVALID_ARG, "chd_graph_begin: capture needs a non-default context stream");
  cudaError_t e = cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, std::string("chd_graph_begin: ") + cudaGetErrorString(e));
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_graph_end(chd_context *ctx, chd_graph **out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(out);
  Context &C = *ctx->c;
  auto *g = new chd_graph();
  cudaError_t e = cudaStreamEndCapture(C.stream, &g->graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    delete g;
    cudaGetLastError();
    return fail(CHD_ERR_CUDA, std::string("chd_graph_end: ") + cudaGetErrorString(e));
  }
  *out = g;
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_graph_launch(chd_context *ctx, const chd_graph *g) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(g);
  cudaError_t e = cudaGraphLaunch(g->exec, ctx->c->stream);
  if (e != cudaSuccess) return fail(CHD_ERR_CUDA, std::string("chd_graph_launch: ") + cudaGetErrorString(e));
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

void chd_graph_destroy(chd_graph *g) { delete g; }

int chd_relinearize(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(key);
  return ctx->c->relinearize(res->ct, a->ct, key->k, false);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_relinearize_rescale(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(key);
  return ctx->c->relinearize(res->ct, a->ct, key->k, true);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_mult_key(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(key);
  return ctx->c->mult_key(res->ct, a->ct, key->k);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hmult(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
              const chd_evk *mult_key, int rescale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(b);
  CHD_NOTNULL(mult_key);
  return ctx->c->hmult(res->ct, a->ct, b->ct, mult_key->k, rescale != 0);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hmult_batch(chd_context *ctx, int count, chd_ciphertext *const *res, const chd_ciphertext *const *a,
                    const chd_ciphertext *const *b, const chd_evk *mult_key, int rescale) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(b);
  CHD_NOTNULL(mult_key);
  if (count < 0) return fail(CHD_ERR_INVALID_ARG, "chd_hmult_batch: negative count");
  std::vector<DeviceCt *> r(count);
  std::vector<const DeviceCt *> x(count), y(count);
  for (int i = 0; i < count; i++) {
    if (!res[i] || !a[i] || !b[i]) return fail(CHD_ERR_INVALID_ARG, "chd_hmult_batch: null ciphertext");
    r[i] = &res[i]->ct;
    x[i] = &a[i]->ct;
    y[i] = &b[i]->ct;
  }
  return ctx->c->hmult_batch(count, r.data(), x.data(), y.data(), mult_key->k, rescale != 0);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hrot(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *rot_key, int rot_dist) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(rot_key);
  return ctx->c->hrot(res->ct, a->ct, rot_key->k, rot_dist);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hconj(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_evk *conj_key) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(conj_key);
  return ctx->c->hconj(res->ct, a->ct, conj_key->k);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hrot_add(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a, const chd_ciphertext *b,
                 const chd_evk *rot_key, int rot_dist) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  CHD_NOTNULL(b);
  CHD_NOTNULL(rot_key);
  return ctx->c->hrot_add(res->ct, a->ct, b->ct, rot_key->k, rot_dist);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_hoisted_rotate(chd_context *ctx, const chd_ciphertext *a, int count, const int *rot_dists,
                       const chd_evk *const *rot_keys, chd_ciphertext *const *out) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(a);
  CHD_NOTNULL(rot_dists);
  CHD_NOTNULL(rot_keys);
  CHD_NOTNULL(out);
  if (count <= 0) return fail(CHD_ERR_INVALID_ARG, "chd_hoisted_rotate: count must be positive");
  std::vector<const DeviceEvk *> k(count);
  std::vector<DeviceCt *> o(count);
  for (int i = 0; i < count; i++) {
    if (!rot_keys[i] || !out[i]) return fail(CHD_ERR_INVALID_ARG, "chd_hoisted_rotate: null key or output");
    k[i] = &rot_keys[i]->k;
    o[i] = &out[i]->ct;
  }
  return ctx->c->hoisted_rotate(a->ct, count, rot_dists, k.data(), o.data());
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_moddown(chd_context *ctx, chd_ciphertext *res, const chd_ciphertext *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  return ctx->c->moddown_ct(res->ct, a->ct);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_moddown_batch(chd_context *ctx, int count, chd_ciphertext *const *res, const chd_ciphertext *const *a) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(res);
  CHD_NOTNULL(a);
  if (count < 1) return fail(CHD_ERR_INVALID_ARG, "chd_moddown_batch: empty batch");
  std::vector<DeviceCt *> r(count);
  std::vector<const DeviceCt *> x(count);
  for (int i = 0; i < count; i++) {
    if (!res[i] || !a[i]) return fail(CHD_ERR_INVALID_ARG, "chd_moddown_batch: null ciphertext");
    r[i] = &res[i]->ct;
    x[i] = &a[i]->ct;
  }
  return ctx->c->moddown_batch(count, r.data(), x.data());
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_ntt(chd_context *ctx, int num_main, int num_ter, int num_aux, uint32_t *data_dev, int mont, int count) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(data_dev);
  CHD_ALIGNED(data_dev);
  NP np{num_main, num_ter, num_aux};
  const Params &P = *ctx->c->P;
  if (num_main < 0 || num_ter < 0 || num_aux < 0 || num_main > P.max_main || num_ter > P.max_ter ||
      num_aux > P.alpha || count < 1)
    return fail(CHD_ERR_INVALID_ARG, "chd_ntt: invalid prime counts");
  return ctx->c->ntt(np, data_dev, mont != 0, count, static_cast<size_t>(np.total()) * P.n);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_intt(chd_context *ctx, int num_main, int num_ter, int num_aux, uint32_t *data_dev, int mont, int count) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(data_dev);
  CHD_ALIGNED(data_dev);
  NP np{num_main, num_ter, num_aux};
  const Params &P = *ctx->c->P;
  if (num_main < 0 || num_ter < 0 || num_aux < 0 || num_main > P.max_main || num_ter > P.max_ter ||
      num_aux > P.alpha || count < 1)
    return fail(CHD_ERR_INVALID_ARG, "chd_intt: invalid prime counts");
  return ctx->c->intt(np, data_dev, mont != 0, count, static_cast<size_t>(np.total()) * P.n);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_modup_raw(chd_context *ctx, int level, const uint32_t *src_dev, uint32_t *dst_dev) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(src_dev);
  CHD_ALIGNED(src_dev);
  CHD_NOTNULL(dst_dev);
  CHD_ALIGNED(dst_dev);
  Context &C = *ctx->c;
  if (level < -1 || level > C.P->max_level) return fail(CHD_ERR_INVALID_LEVEL, "chd_modup_raw: invalid level");
  const LevelMS &m = C.lms(level);
  const size_t stride = static_cast<size_t>(m.num_q + m.num_aux) * C.P->n;
  std::vector<uint32_t *> d(m.beta);
  for (int i = 0; i < m.beta; i++) d[i] = dst_dev + i * stride;
  return C.modup(level, src_dev, d.data());
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_moddown_raw(chd_context *ctx, int level, int type, const uint32_t *src_dev, uint32_t *dst_dev, int npoly) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(src_dev);
  CHD_ALIGNED(src_dev);
  CHD_NOTNULL(dst_dev);
  CHD_ALIGNED(dst_dev);
  Context &C = *ctx->c;
  if (level < -1 || level > C.P->max_level) return fail(CHD_ERR_INVALID_LEVEL, "chd_moddown_raw: invalid level");
  if (type < 0 || type > 2 || npoly < 1) return fail(CHD_ERR_INVALID_ARG, "chd_moddown_raw: bad type or npoly");
  if (type != CHD_MODDOWN && level < 1) return fail(CHD_ERR_INVALID_LEVEL, "chd_moddown_raw: cannot rescale");
  const LevelMS &m = C.lms(level);
  const int nsa = type == CHD_RESCALE ? 0 : m.num_aux;
  NP ns = C.P->level_np(level, nsa);
  NP nd = C.P->level_np(type == CHD_MODDOWN ? level : level - 1, 0);
  std::vector<const uint32_t *> s(npoly);
  std::vector<uint32_t *> d(npoly);
  for (int p = 0; p < npoly; p++) {
    s[p] = src_dev + static_cast<size_t>(p) * ns.total() * C.P->n;
    d[p] = dst_dev + static_cast<size_t>(p) * nd.total() * C.P->n;
  }
  Context::MDType t = type == CHD_MODDOWN ? Context::MDType::kModDown
                      : type == CHD_RESCALE ? Context::MDType::kRescale : Context::MDType::kModDownRescale;
  return C.moddown(level, t, s.data(), d.data(), npoly);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

namespace {
// BConv table of ModSwitchMatrixMult (ModSwitch.cu:320-411): T[m][k] =
// centre(prod_{j != k} src_j * R^2 mod dst_m), validated indices
int bconv_table(const Context &C, const int *src_gidx, int K, const int *dst_gidx, int M, std::vector<int32_t> *t,
                const char *who) {
  const int np_all = C.P->L + C.P->alpha;
  if (K < 1 || K > 16 || M < 1 || M > 64) return fail(CHD_ERR_UNSUPPORTED, std::string(who) + ": K in [1,16], M in [1,64]");
  for (int i = 0; i < K; i++)
    if (src_gidx[i] < 0 || src_gidx[i] >= np_all) return fail(CHD_ERR_INVALID_ARG, std::string(who) + ": bad src index");
  for (int i = 0; i < M; i++)
    if (dst_gidx[i] < 0 || dst_gidx[i] >= np_all) return fail(CHD_ERR_INVALID_ARG, std::string(who) + ": bad dst index");
  t->assign(static_cast<size_t>(M) * K, 0);
  for (int m = 0; m < M; m++) {
    uint32_t p = C.P->primes[dst_gidx[m]];
    for (int k = 0; k < K; k++) {
      uint32_t acc = 1;
      for (int j = 0; j < K; j++)
        if (j != k) acc = prime::mul_mod(acc, C.P->primes[src_gidx[j]], p);
      (*t)[m * K + k] = prime::centre(prime::to_mont(prime::to_mont(acc, p), p), p);
    }
  }
  return CHD_OK;
}
}  // namespace

int chd_bconv_raw(chd_context *ctx, const int32_t *xt_dev, const int *src_gidx, int K, const int *dst_gidx, int M,
                  uint32_t *out_dev) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(xt_dev);
  CHD_ALIGNED(xt_dev);
  CHD_NOTNULL(src_gidx);
  CHD_NOTNULL(dst_gidx);
  CHD_NOTNULL(out_dev);
  CHD_ALIGNED(out_dev);
  Context &C = *ctx->c;
  std::vector<int32_t> t;
  int rc = bconv_table(C, src_gidx, K, dst_gidx, M, &t, "chd_bconv_raw");
  if (rc != CHD_OK) return rc;
  int32_t *dt = nullptr;
  if (cudaMalloc(&dt, t.size() * 4) != cudaSuccess) return fail(CHD_ERR_ALLOC, "chd_bconv_raw: allocation failed");
  cudaMemcpyAsync(dt, t.data(), t.size() * 4, cudaMemcpyHostToDevice, C.stream);
  rc = C.bconv(xt_dev, K, dt, dst_gidx, M, out_dev);
  cudaStreamSynchronize(C.stream);
  cudaFree(dt);
  return rc;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_bconv_batch(chd_context *ctx, int engine, int npoly, const int32_t *xt_dev, const int *src_gidx, int K,
                    const int *dst_gidx, int M, uint32_t *out_dev) try {
  CHD_CTX(ctx);
  CHD_NOTNULL(src_gidx);
  CHD_NOTNULL(dst_gidx);
  if (npoly < 0) return fail(CHD_ERR_INVALID_ARG, "chd_bconv_batch: negative npoly");
  if (npoly > 0 && (!xt_dev || !out_dev)) return fail(CHD_ERR_INVALID_ARG, "chd_bconv_batch: null buffer");
  if (engine != CHD_BCONV_CUDA_CORE && engine != CHD_BCONV_TENSOR_CORE)
    return fail(CHD_ERR_INVALID_ARG, "chd_bconv_batch: unknown engine");
  Context &C = *ctx->c;
  std::vector<int32_t> t;
  int rc = bconv_table(C, src_gidx, K, dst_gidx, M, &t, "chd_bconv_batch");
  if (rc != CHD_OK) return rc;
  return C.bconv_many(engine, npoly, xt_dev, K, t, dst_gidx, M, out_dev);
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

int chd_params_level_consts(const char *json_text, int level, int kind, int digit, uint32_t *c1, int32_t *table,
                            uint32_t *inv, uint32_t *pad, int *dims) try {
  CHD_NOTNULL(json_text);
  CHD_NOTNULL(dims);
  ParamSpec spec;
  std::string err;
  if (!parse_param_json(json_text, &spec, &err)) return fail(CHD_ERR_PARSE, err);
  auto P = Params::create(spec, &err);
  if (!P) return fail(CHD_ERR_INVALID_ARG, err);
  if (level < -1 || level > P->max_level) return fail(CHD_ERR_INVALID_LEVEL, "invalid level");
  LevelMS m;
  build_level_ms(*P, level, &m);
  const std::vector<uint32_t> *v1 = nullptr, *vi = nullptr, *vp = nullptr;
  const std::vector<int32_t> *vt = nullptr;
  int K = 0, M = 0;
  dims[3] = m.restore_start;
  dims[4] = m.restore_end;
  dims[5] = m.beta;
  switch (kind) {
    case 0: {  // ModUp digit
      if (digit < 0 || digit >= m.beta) return fail(CHD_ERR_INVALID_ARG, "invalid digit");
      K = m.dig_e[digit] - m.dig_s[digit];
      if (K <= 0) {
        dims[0] = dims[1] = dims[2] = 0;
        return CHD_OK;
      }
      M = m.num_q + m.num_aux - K;
      for (int i = 0; i < K; i++) c1[i] = m.mod_up1[m.dig_s[digit] + i];
      vt = &m.mod_up2[digit];
      break;
    }
    case 1:
      v1 = &m.mod_down1, vt = &m.mod_down2, vi = &m.inv_p_prod;
      K = m.num_aux, M = m.num_q;
      break;
    case 2:
    case 3:
      if (!m.has_rescale) return fail(CHD_ERR_INVALID_LEVEL, "no rescale at this level");
      v1 = kind == 2 ? &m.rs1 : &m.mdr1;
      vt = kind == 2 ? &m.rs2 : &m.mdr2;
      vi = kind == 2 ? &m.rs_inv : &m.mdr_inv;
      vp = kind == 2 ? &m.rs_pad : &m.mdr_pad;
      K = kind == 2 ? m.rs_src_len : m.mdr_src_len;
      M = m.rs_dst_len;
      break;
    default:
      return fail(CHD_ERR_INVALID_ARG, "invalid kind");
  }
  dims[0] = K;
  dims[1] = M;
  dims[2] = vp ? static_cast<int>(vp->size()) : 0;
  if (v1 && c1) std::copy(v1->begin(), v1->end(), c1);
  if (vt && table) std::copy(vt->begin(), vt->end(), table);
  if (vi && inv) std::copy(vi->begin(), vi->end(), inv);
  if (vp && pad) std::copy(vp->begin(), vp->end(), pad);
  return CHD_OK;
} catch (const std::exception &e) {
  return fail(CHD_ERR_INTERNAL, std::string("internal error: ") + e.what());
} catch (...) {
  return fail(CHD_ERR_INTERNAL, "internal error");
}

}  // extern "C"
