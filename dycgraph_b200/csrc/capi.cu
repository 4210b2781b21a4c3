// capi.cu -- extern "C" entry points declared in include/dycg.h. Every entry
// point converts exceptions into a status code; nothing aborts the process.
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "engine.h"

using dycg::Engine;
using dycg::Error;

struct dycg_engine {
  Engine *impl;
  std::string error;
};

namespace {

// Runs f on the engine and turns exceptions into status codes. join: the
// engine stream first waits for side-stream page staging of an earlier call;
// the snapshot calls pass false and join after their ingest instead.
template <class F>
int guard(dycg_engine *e, F &&f, bool join = true) {
  if (!e || !e->impl) return DYCG_EINVAL;
  try {
    if (join) e->impl->join();
    f(*e->impl);
    return DYCG_OK;
  } catch (const Error &x) {
    e->error = x.what();
    return x.code;
  } catch (const std::bad_alloc &) {
    e->error = "host allocation failed";
    return DYCG_ENOMEM;
  } catch (const std::exception &x) {
    e->error = x.what();
    return DYCG_EINVAL;
  }
}

}  // namespace

extern "C" {

int dycg_options_default(dycg_options *opt) {
  if (!opt) return DYCG_EINVAL;
  std::memset(opt, 0, sizeof(*opt));
  opt->algo = DYCG_ALGO_SSSP;
  opt->weight_mode = DYCG_WEIGHT_HASH128;
  opt->source = 0;
  opt->segments = 1;
  opt->hbm_graph_budget_bytes = 0;
  opt->cache_policy = DYCG_CACHE_NONE;
  opt->symmetric = 0;
  opt->epsilon = 1e-6f;
  opt->alpha = 0.85f;
  opt->max_rounds = 100;
  opt->device = 0;
  opt->page_shift = 12;
  return DYCG_OK;
}

int dycg_create(const dycg_options *opt, dycg_engine **out) {
  if (!opt || !out) return DYCG_EINVAL;
  *out = nullptr;
  dycg_engine *e = new (std::nothrow) dycg_engine();
  if (!e) return DYCG_ENOMEM;
  try {
    e->impl = new Engine(*opt);
  } catch (const Error &x) {
    int code = x.code;
    delete e;
    std::fprintf(stderr, "dycg_create: %s\n", x.what());
    return code;
  } catch (const std::exception &x) {
    delete e;
    std::fprintf(stderr, "dycg_create: %s\n", x.what());
    return DYCG_ECUDA;
  }
  *out = e;
  return DYCG_OK;
}

void dycg_destroy(dycg_engine *e) {
  if (!e) return;
  delete e->impl;
  delete e;
}

int dycg_load_graph_csr(dycg_engine *e, uint32_t n, const uint64_t *offsets, const uint32_t *dst,
                        const uint32_t *w) {
  return guard(e, [&](Engine &g) { g.load_csr(n, offsets, dst, w); });
}

int dycg_load_graph_file(dycg_engine *e, const char *path, uint32_t min_nodes, int weighted) {
  if (!path) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.load_file(path, min_nodes, weighted); });
}

int dycg_load_graph_binary(dycg_engine *e, const char *path) {
  if (!path) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.load_binary(path); });
}

int dycg_load_graph_rmat(dycg_engine *e, uint32_t scale, uint32_t edge_factor, double a, double b,
                         double c, uint64_t seed, uint32_t wlo, uint32_t whi, int symmetrize) {
  return guard(e, [&](Engine &g) { g.load_rmat(scale, edge_factor, a, b, c, seed, wlo, whi, symmetrize); });
}

int dycg_load_graph_grid(dycg_engine *e, uint32_t side, uint32_t shortcut_permille, uint32_t radius,
                         uint64_t seed, uint32_t wlo, uint32_t whi) {
  return guard(e, [&](Engine &g) { g.load_grid(side, shortcut_permille, radius, seed, wlo, whi); });
}

int dycg_init(dycg_engine *e) {
  return guard(e, [&](Engine &g) { g.init(); });
}

int dycg_delete_edges(dycg_engine *e, const dycg_edge *dels, size_t nd, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.apply(dels, nd, nullptr, 0, false, 1, false, stats); }, false);
}

int dycg_insert_edges(dycg_engine *e, const dycg_edge *adds, size_t na, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.apply(nullptr, 0, adds, na, false, 2, false, stats); }, false);
}

int dycg_cache_maintenance(dycg_engine *e, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.cache_maintenance(false, stats); });
}

int dycg_reserve_batch(dycg_engine *e, size_t max_records) {
  return guard(e, [&](Engine &g) { g.reserve_batch(max_records); });
}

int dycg_apply_batch(dycg_engine *e, const dycg_edge *dels, size_t nd, const dycg_edge *adds,
                     size_t na, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.apply(dels, nd, adds, na, false, 0, true, stats); }, false);
}

int dycg_apply_batch_device(dycg_engine *e, const dycg_edge *d_dels, size_t nd,
                            const dycg_edge *d_adds, size_t na, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.apply(d_dels, nd, d_adds, na, true, 0, true, stats); }, false);
}

int dycg_gather(dycg_engine *e, uint32_t *values, uint32_t *parents) {
  return guard(e, [&](Engine &g) { g.gather(values, parents); });
}

int dycg_gather_ranks(dycg_engine *e, float *ranks, float *residuals) {
  return guard(e, [&](Engine &g) { g.gather_ranks(ranks, residuals); });
}

int dycg_get_row(dycg_engine *e, uint32_t v, int incoming, uint32_t *dst, uint32_t *w, uint32_t cap,
                 uint32_t *deg) {
  return guard(e, [&](Engine &g) { g.get_row(v, incoming, dst, w, cap, deg); });
}

int dycg_export_csr(dycg_engine *e, uint64_t *offsets, uint32_t *dst, uint32_t *w) {
  if (!offsets) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.export_csr(offsets, dst, w); });
}

int dycg_graph_info_get(dycg_engine *e, dycg_graph_info *info) {
  if (!info) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.info(info); });
}

int dycg_sample_edges(dycg_engine *e, uint64_t count, uint64_t seed, dycg_edge *out) {
  if (!out && count) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.sample_edges(count, seed, out); });
}

int dycg_gen_rmat_edges(uint32_t scale, double a, double b, double c, uint64_t seed, uint64_t first,
                        uint64_t count, uint32_t wlo, uint32_t whi, dycg_edge *out) {
  if ((!out && count) || scale < 1 || scale > 31 || wlo == 0 || whi < wlo) return DYCG_EINVAL;
  const double S = (double)(1u << 21);
  const uint32_t ta = (uint32_t)(a * S), tab = (uint32_t)((a + b) * S),
                 tabc = (uint32_t)((a + b + c) * S);
  const uint64_t wseed = seed ^ 0x5745494748545321ull;
  for (uint64_t i = 0; i < count; i++) {
    uint32_t u, v;
    dycg::rmat_draw(seed, first + i, scale, ta, tab, tabc, u, v);
    out[i].u = u;
    out[i].v = v;
    out[i].w = dycg::hash_weight(wseed, u, v, wlo, whi);
  }
  return DYCG_OK;
}

int dycg_convert_graph_text(const char *text_path, const char *binary_path, uint32_t min_nodes,
                            int weighted) {
  if (!text_path || !binary_path) return DYCG_EINVAL;
  try {
    const dycg::TextGraph g = dycg::parse_text_graph(text_path, min_nodes, weighted);
    std::FILE *f = std::fopen(binary_path, "wb");
    if (!f) return DYCG_EIO;
    const uint64_t hdr[3] = {g.n, g.m, weighted ? 1ull : 0ull};
    bool ok = std::fwrite("DYCGCSR1", 1, 8, f) == 8 && std::fwrite(hdr, 8, 3, f) == 3 &&
              std::fwrite(g.off.data(), 8, g.n + 1ull, f) == g.n + 1ull &&
              std::fwrite(g.dst.data(), 4, g.m, f) == g.m &&
              (!weighted || std::fwrite(g.w.data(), 4, g.m, f) == g.m);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? DYCG_OK : DYCG_EIO;
  } catch (const Error &x) {
    return x.code;
  } catch (const std::bad_alloc &) {
    return DYCG_ENOMEM;
  } catch (const std::exception &) {
    return DYCG_EINVAL;
  }
}

uint32_t dycg_hash_weight(uint64_t seed, uint32_t u, uint32_t v, uint32_t wlo, uint32_t whi) {
  if (whi < wlo) return wlo;
  return dycg::hash_weight(seed ^ 0x5745494748545321ull, u, v, wlo, whi);
}

int dycg_set_queries(dycg_engine *e, const uint32_t *sources, uint32_t count, uint32_t mode) {
  if (!sources && count) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.set_queries(sources, count, mode); });
}

int dycg_set_query_mapping(dycg_engine *e, uint32_t qratio, uint32_t heavy, uint32_t tile) {
  return guard(e, [&](Engine &g) { g.set_query_mapping(qratio, heavy, tile); });
}

int dycg_set_query_queue(dycg_engine *e, uint32_t scheme) {
  return guard(e, [&](Engine &g) { g.set_query_queue(scheme); });
}

int dycg_gather_query(dycg_engine *e, uint32_t q, uint32_t *values, uint32_t *parents) {
  return guard(e, [&](Engine &g) { g.gather_query(q, values, parents); });
}

int dycg_tune_query_mapping(dycg_engine *e, const dycg_edge *dels, size_t nd,
                            const dycg_edge *adds, size_t na, dycg_query_mapping *tried,
                            uint32_t cap, uint32_t *n_tried, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) { g.tune(dels, nd, adds, na, tried, cap, n_tried, stats); });
}

int dycg_apply_batches(dycg_engine *e, const dycg_edge *dels, const uint64_t *del_counts,
                       const dycg_edge *adds, const uint64_t *add_counts, uint32_t snapshots,
                       dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) {
    g.apply_batches(dels, del_counts, adds, add_counts, snapshots, false, stats);
  });
}

int dycg_apply_batches_device(dycg_engine *e, const dycg_edge *d_dels, const uint64_t *del_counts,
                              const dycg_edge *d_adds, const uint64_t *add_counts,
                              uint32_t snapshots, dycg_batch_stats *stats) {
  return guard(e, [&](Engine &g) {
    g.apply_batches(d_dels, del_counts, d_adds, add_counts, snapshots, true, stats);
  });
}

int dycg_set_cache_policy(dycg_engine *e, uint32_t policy) {
  return guard(e, [&](Engine &g) { g.set_cache_policy(policy); });
}

int dycg_policy_trace(dycg_engine *e, uint32_t snapshots) {
  return guard(e, [&](Engine &g) { g.policy_trace(snapshots); });
}

int dycg_policy_train(dycg_engine *e, uint32_t epochs, float lr, uint32_t batch, uint64_t seed,
                      dycg_policy_report *report) {
  return guard(e, [&](Engine &g) { g.policy_train(epochs, lr, batch, seed, report); });
}

int dycg_policy_params(dycg_engine *e, float *params) {
  if (!params) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.policy_params(params); });
}

int dycg_policy_set_params(dycg_engine *e, const float *params) {
  if (!params) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.policy_set_params(params); });
}

int dycg_mlp_infer(const void *d_x, uint32_t n, const float *d_params, float *d_out,
                   void *stream) {
  if ((!d_x || !d_out) && n) return DYCG_EINVAL;
  if (!d_params) return DYCG_EINVAL;
  if (!n) return DYCG_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (dycg::launch_mlp_infer(d_x, n, d_params, d_out, nullptr, nullptr, s) != cudaSuccess)
    return DYCG_ECUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? DYCG_OK : DYCG_ECUDA;
}

int dycg_mlp_loss_grad(const void *d_x, const float *d_y, uint32_t n, const float *d_params,
                       float *d_grad, float *d_loss, void *stream) {
  if ((!d_x || !d_y) && n) return DYCG_EINVAL;
  if (!d_params || !d_grad || !d_loss) return DYCG_EINVAL;
  if (!n) return DYCG_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (dycg::launch_mlp_grad(d_x, d_y, n, n, 0, d_params, 2.f, d_grad, d_loss, nullptr, s) !=
      cudaSuccess)
    return DYCG_ECUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? DYCG_OK : DYCG_ECUDA;
}

int dycg_sample_row_edges(dycg_engine *e, const uint32_t *sources, uint64_t count, uint64_t seed,
                          dycg_edge *out) {
  if ((!sources || !out) && count) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { g.sample_row_edges(sources, count, seed, out); });
}

int dycg_stream(dycg_engine *e, void **stream) {
  if (!stream) return DYCG_EINVAL;
  return guard(e, [&](Engine &g) { *stream = (void *)g.stream(); });
}

int dycg_last_error(dycg_engine *e, char *buf, size_t len) {
  if (!e || !buf || !len) return DYCG_EINVAL;
  std::snprintf(buf, len, "%s", e->error.c_str());
  return DYCG_OK;
}

const char *dycg_version(void) { return "dycg-b200 0.1.0 (sm_100a)"; }

}  // extern "C"
