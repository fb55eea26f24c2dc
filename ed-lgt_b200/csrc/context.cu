// Tuning context: an explicit, caller-owned store of autotuner choices
// (launch shapes keyed by a hash of the problem shape).  The library keeps no
// global mutable state for tuning; every tuned entry point's caller passes the
// parameters it read from a context it created.
#include "internal.cuh"

#include <mutex>
#include <new>
#include <unordered_map>
#include <vector>

struct edg_ctx {
  std::mutex mu;
  std::unordered_map<uint64_t, std::vector<int32_t>> entries;
};

extern "C" edg_ctx* edg_ctx_create(void) { return new (std::nothrow) edg_ctx(); }

extern "C" void edg_ctx_destroy(edg_ctx* ctx) { delete ctx; }

extern "C" int edg_ctx_put(edg_ctx* ctx, uint64_t key, const int32_t* params, int32_t n_params) {
  EDG_REQUIRE(ctx != nullptr, "edg_ctx_put: null context");
  EDG_REQUIRE(n_params >= 1 && n_params <= EDG_CTX_MAX_PARAMS && params != nullptr,
              "edg_ctx_put: need 1..%d parameters", EDG_CTX_MAX_PARAMS);
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->entries[key] = std::vector<int32_t>(params, params + n_params);
  return EDG_OK;
}

extern "C" int edg_ctx_get(edg_ctx* ctx, uint64_t key, int32_t* params, int32_t n_params) {
  EDG_REQUIRE(ctx != nullptr && params != nullptr, "edg_ctx_get: null pointer");
  std::lock_guard<std::mutex> lock(ctx->mu);
  auto it = ctx->entries.find(key);
  if (it == ctx->entries.end()) return 0;
  const int32_t n = (int32_t)it->second.size() < n_params ? (int32_t)it->second.size() : n_params;
  for (int32_t i = 0; i < n; ++i) params[i] = it->second[i];
  return n;
}

extern "C" int64_t edg_ctx_size(edg_ctx* ctx) {
  if (ctx == nullptr) return -1;
  std::lock_guard<std::mutex> lock(ctx->mu);
  return (int64_t)ctx->entries.size();
}
