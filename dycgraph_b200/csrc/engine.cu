// engine.cu -- host orchestration of the B200 delta-repair engine.
//
// The Engine mirrors the reference's sepgraph::engine::Engine
// (include/framework/framework.cuh:780-6112) for one path: load a graph into
// the paged pinned store, solve once, then per snapshot ingest + mutate +
// repair + cache maintenance, all on one CUDA stream with one host
// synchronisation at the end of a batch (two when the cache refreshes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_set>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "engine.h"

namespace dycg {

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t _e = (x);                                                                  \
    if (_e != cudaSuccess)                                                                 \
      throw Error(_e == cudaErrorMemoryAllocation ? DYCG_ENOMEM : DYCG_ECUDA,              \
                  std::string(#x) + ": " + cudaGetErrorString(_e));                        \
  } while (0)

static u64 round_up(u64 x, u64 m) { return (x + m - 1) / m * m; }
static void fill_phases(dycg_batch_stats *s, const Ctl &c);

Engine::Engine(const dycg_options &opt) : opt_(opt) {
  if (opt_.algo > DYCG_ALGO_PR) throw Error(DYCG_EINVAL, "unknown algorithm");
  if (opt_.page_shift == 0) opt_.page_shift = 12;
  if (opt_.page_shift < 8 || opt_.page_shift > 20) throw Error(DYCG_EINVAL, "page_shift out of range");
  if (opt_.max_rounds == 0) opt_.max_rounds = 100;
  if (!(opt_.alpha > 0.f && opt_.alpha < 1.f)) opt_.alpha = 0.85f;
  page_shift_ = opt_.page_shift;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw Error(DYCG_ENOGPU, "no CUDA device available");
  dev_ = opt_.device;
  if (dev_ < 0 || dev_ >= ndev) throw Error(DYCG_EINVAL, "device ordinal out of range");
  CK(cudaSetDevice(dev_));
  CK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev_));
  int coop = 0;
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev_));
  if (!coop) throw Error(DYCG_ENOGPU, "device lacks cooperative launch");
  CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&fst_, cudaStreamNonBlocking));
  for (auto &e : ev_) CK(cudaEventCreate(&e));
  for (auto &e : fev_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (opt_.cache_policy > DYCG_CACHE_LEARNED) throw Error(DYCG_EINVAL, "unknown cache policy");
  if (opt_.frontier_queue > DYCG_QUEUE_CLAIMED)
    throw Error(DYCG_EINVAL, "unknown frontier-queue scheme");
  // one CTA per SM: 2.64 ms of mutation per 100K-update R-MAT 26 snapshot,
  // against 2.85 ms with one warp per record (same box and snapshots)
  mut_ctas_ = opt_.mutation_ctas ? opt_.mutation_ctas : (uint32_t)num_sms_;
  policy_ = opt_.cache_policy;
  stored_ = opt_.algo == DYCG_ALGO_SSSP && opt_.weight_mode == DYCG_WEIGHT_STORED;
  has_in_ = !opt_.symmetric && opt_.algo != DYCG_ALGO_PR;
}

Engine::~Engine() {
  if (fst_) cudaStreamSynchronize(fst_);
  if (st_) cudaStreamSynchronize(st_);
  drop_graphs();
  for (cudaEvent_t e : bev_) cudaEventDestroy(e);
  if (h_rec_) cudaFreeHost(h_rec_);
  if (d_rec_) cudaFree(d_rec_);
  if (h_bctl_) cudaFreeHost(h_bctl_);
  for (void *p : {(void *)dbufs_.k_in, (void *)dbufs_.k_out, (void *)dbufs_.v_in,
                  (void *)dbufs_.v_out, dbufs_.temp})
    cudaFree(p);
  if (tx_) cudaFree(tx_);
  if (ty_) cudaFree(ty_);
  for (auto &e : pev_)
    if (e) cudaEventDestroy(e);
  dfree_all();
  for (void *p : hallocs_) cudaFreeHost(p);
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  for (auto &e : fev_)
    if (e) cudaEventDestroy(e);
  if (fst_) cudaStreamDestroy(fst_);
  if (st_) cudaStreamDestroy(st_);
}

void Engine::join_staging() {
  if (!staging_) return;
  CK(cudaStreamWaitEvent(st_, fev_[1], 0));
  staging_ = false;
}

void *Engine::dmalloc(size_t bytes) {
  void *p = nullptr;
  CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
  dallocs_.push_back(p);
  return p;
}

void Engine::dfree_all() {
  for (void *p : dallocs_) cudaFree(p);
  dallocs_.clear();
  for (void *p : batch_allocs_) cudaFree(p);
  batch_allocs_.clear();
}

void Engine::sync_check(const char *where) {
  CK(cudaStreamSynchronize(st_));
  CK(cudaGetLastError());
  (void)where;
}

void Engine::check_loaded() const {
  if (!loaded_) throw Error(DYCG_ESTATE, "no graph loaded");
}

Adj Engine::adj(const Arena &A) const {
  Adj a;
  a.hdst = A.d_dst;
  a.cdst = cdst_;
  a.stride = A.stride;
  a.fence_shift = A.fence_shift;
  a.tbits = A.tbits;
  a.page_slot = page_slot_;
  a.page_hits = page_hits_;
  a.page_base = A.page_base;
  a.page_shift = page_shift_;
  a.off = A.off;
  a.len = A.len;
  a.cap = A.cap;
  a.srt = A.srt;
  a.live = A.live;
  a.top = A.top;
  a.arena = A.slots;
  a.fence = A.fence;
  return a;
}

// ---- graph construction ---------------------------------------------------

// keys: sorted (row << 32 | neighbour), m of them, no KEY_INF among them.
void Engine::build_direction(Arena &A, const u64 *keys, const uint32_t *wv, u64 m,
                             bool weight_from_hash, u64 wseed, uint32_t wlo, uint32_t whi,
                             bool swapped) {
  const uint32_t n = n_;
  uint32_t *deg = (uint32_t *)dmalloc((n + 1ull) * 4);
  u64 *cap64 = (u64 *)dmalloc((n + 1ull) * 8);
  u64 *rowstart = (u64 *)dmalloc((n + 1ull) * 8);
  CK(cudaMemsetAsync(deg, 0, (n + 1ull) * 4, st_));
  CK(cudaMemsetAsync(cap64, 0, (n + 1ull) * 8, st_));
  A.off = (u64 *)dmalloc((n + 1ull) * 8);
  A.len = (uint32_t *)dmalloc((n + 1ull) * 4);
  A.cap = (uint32_t *)dmalloc((n + 1ull) * 4);
  A.srt = (uint32_t *)dmalloc((n + 1ull) * 4);
  A.live = (uint32_t *)dmalloc((n + 1ull) * 4);
  A.top = (u64 *)dmalloc(8);
  CK(build_degrees(keys, m, deg, st_));
  CK(build_caps(deg, n, cap64, A.cap, A.len, A.srt, A.live, st_));
  size_t tb = 0;
  CK(build_scan_u64(nullptr, tb, cap64, A.off, n + 1ull, st_));
  size_t tb2 = 0;
  CK(build_scan_u32_to_u64(nullptr, tb2, deg, rowstart, n + 1ull, st_));
  void *temp = dmalloc(std::max(tb, tb2));
  CK(build_scan_u64(temp, tb, cap64, A.off, n + 1ull, st_));
  CK(build_scan_u32_to_u64(temp, tb2, deg, rowstart, n + 1ull, st_));
  u64 total = 0;
  CK(cudaMemcpyAsync(&total, A.off + n, 8, cudaMemcpyDeviceToHost, st_));
  sync_check("layout");
  const u64 page = 1ull << page_shift_;
  const u64 permille = opt_.arena_headroom_permille ? opt_.arena_headroom_permille : 125;
  const u64 head = std::max<u64>(total / 1000 * permille, 1ull << 20);
  A.slots = round_up(total + head, page);
  A.pages = (uint32_t)(A.slots >> page_shift_);
  A.stride = stored_ ? 2 : 1;
  A.fence_shift = stored_ ? 4 : 5;
  void *hd = nullptr;
  CK(cudaHostAlloc(&hd, A.slots * 4 * A.stride, cudaHostAllocMapped | cudaHostAllocPortable));
  hallocs_.push_back(hd);
  A.h_dst = (uint32_t *)hd;
  CK(cudaHostGetDevicePointer((void **)&A.d_dst, hd, 0));
  A.fence = (uint32_t *)dmalloc((A.slots >> A.fence_shift) * 4);
  A.tbits = (uint32_t *)dmalloc((A.slots >> 5) * 4);
  CK(cudaMemsetAsync(A.tbits, 0, (A.slots >> 5) * 4, st_));
  CK(cudaMemcpyAsync(A.top, &total, 8, cudaMemcpyHostToDevice, st_));
  CK(build_scatter(keys, wv, m, A.off, rowstart, A.d_dst, A.stride, A.fence, A.fence_shift, wseed,
                   wlo, whi, weight_from_hash ? 1 : 0, swapped ? 1 : 0, st_));
  sync_check("scatter");
  // free the temporaries (they are the last allocations made)
  for (void *p : {temp, (void *)rowstart, (void *)cap64, (void *)deg}) {
    auto it = std::find(dallocs_.begin(), dallocs_.end(), p);
    if (it != dallocs_.end()) dallocs_.erase(it);
    cudaFree(p);
  }
}

// keys/wv: device arrays holding m sorted out-keys (and weights); scratch
// buffers of the same size are used to build the incoming direction.
void Engine::build_from_sorted_keys(u64 *keys, uint32_t *wv, u64 m, bool weight_from_hash,
                                    u64 wseed, uint32_t wlo, uint32_t whi, u64 *scratch_keys,
                                    uint32_t *scratch_w) {
  build_direction(out_, keys, wv, m, weight_from_hash, wseed, wlo, whi, false);
  if (has_in_) {
    CK(build_swap_keys(keys, scratch_keys, m, st_));
    size_t tb = 0;
    CK(build_sort(nullptr, tb, scratch_keys, keys, wv ? wv : nullptr, wv ? scratch_w : nullptr, m,
                  st_));
    void *temp = nullptr;
    CK(cudaMalloc(&temp, std::max<size_t>(tb, 16)));
    // wv holds the weights in out-key order; sort them along with the swapped keys
    cudaError_t e = build_sort(temp, tb, scratch_keys, keys, wv ? wv : nullptr,
                               wv ? scratch_w : nullptr, m, st_);
    cudaStreamSynchronize(st_);
    cudaFree(temp);
    CK(e);
    build_direction(in_, keys, wv ? scratch_w : nullptr, m, weight_from_hash, wseed, wlo, whi,
                    true);
    in_.page_base = out_.pages;
  }
  finish_load();
}

void Engine::finish_load() {
  const uint32_t n = n_;
  npages_ = out_.pages + (has_in_ ? in_.pages : 0);
  page_slot_ = (uint32_t *)dmalloc((u64)npages_ * 4);
  page_hits_ = (uint32_t *)dmalloc((u64)npages_ * 4);
  CK(cudaMemsetAsync(page_slot_, 0xFF, (u64)npages_ * 4, st_));
  CK(cudaMemsetAsync(page_hits_, 0, (u64)npages_ * 4, st_));
  // the HBM graph budget covers the fence index, the deletion bitmap and the
  // cached pages
  const u64 page_bytes = (4ull << page_shift_) * out_.stride;
  const u64 index_bytes =
      ((out_.slots >> out_.fence_shift) + (out_.slots >> 5)) * 4 +
      (has_in_ ? ((in_.slots >> in_.fence_shift) + (in_.slots >> 5)) * 4 : 0);
  index_bytes_ = index_bytes;
  const u64 avail = opt_.hbm_graph_budget_bytes > index_bytes ? opt_.hbm_graph_budget_bytes - index_bytes : 0;
  u64 slots = opt_.cache_policy == DYCG_CACHE_NONE ? 0 : avail / page_bytes;
  slots = std::min<u64>(slots, npages_);
  cache_slots_ = (uint32_t)slots;
  if (cache_slots_) {
    cdst_ = (uint32_t *)dmalloc(((u64)cache_slots_ << page_shift_) * 4 * out_.stride);
    free_list_ = (uint32_t *)dmalloc((u64)cache_slots_ * 4);
    std::vector<uint32_t> fl(cache_slots_);
    for (uint32_t i = 0; i < cache_slots_; i++) fl[i] = cache_slots_ - 1 - i;
    CK(cudaMemcpyAsync(free_list_, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, st_));
    cwk_.hits = page_hits_;
    cwk_.score = (float *)dmalloc((u64)npages_ * 4);
    cwk_.score_sorted = (float *)dmalloc((u64)npages_ * 4);
    cwk_.ids = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.ids_sorted = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.fa = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.fe = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.sa = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.se = (uint32_t *)dmalloc((u64)npages_ * 4);
    cwk_.admit = (uint32_t *)dmalloc((u64)npages_ * 4);
    CK(cudaMemsetAsync(cwk_.score, 0, (u64)npages_ * 4, st_));
    cwk_.temp_bytes = cache_temp_bytes(npages_);
    cwk_.temp = dmalloc(cwk_.temp_bytes);
    cwk_.plan = (CachePlan *)dmalloc(sizeof(CachePlan));
    void *hc = nullptr;
    CK(cudaHostAlloc(&hc, sizeof(CachePlan), cudaHostAllocDefault));
    hallocs_.push_back(hc);
    cwk_.h_plan = (CachePlan *)hc;
    std::memset(cwk_.h_plan, 0, sizeof(CachePlan));
    cwk_.h_plan->free_count = cache_slots_;
    CK(cudaMemcpyAsync(cwk_.plan, cwk_.h_plan, sizeof(CachePlan), cudaMemcpyHostToDevice, st_));
  }
  // vertex state
  key_ = (u64 *)dmalloc((n + 1ull) * 8);
  mark_ = (uint32_t *)dmalloc((n + 1ull) * 4);
  wtag_ = (uint32_t *)dmalloc((n + 1ull) * 4);
  touch_ = (uint32_t *)dmalloc((n + 1ull) * 4);
  aff_ = (uint32_t *)dmalloc((n + 1ull) * 4);
  // wave queues: n + 64 entries, enough for the batched form's 64
  // range-ordered regions of ceil(n / 64) entries each
  q0_ = (uint32_t *)dmalloc((n + 64ull) * 4);
  q1_ = (uint32_t *)dmalloc((n + 64ull) * 4);
  q2_ = opt_.ordered_delta ? (uint32_t *)dmalloc((n + 1ull) * 4) : nullptr;
  CK(cudaMemsetAsync(mark_, 0, (n + 1ull) * 4, st_));
  CK(cudaMemsetAsync(wtag_, 0, (n + 1ull) * 4, st_));
  CK(cudaMemsetAsync(touch_, 0, (n + 1ull) * 4, st_));
  const u64 maxslots = std::max(out_.slots, in_.slots);
  const u64 tcap = maxslots / TILE + maxslots / HEAVY + 4096;
  tile_cap_ = (uint32_t)std::min<u64>(tcap, 0x7FFFFFFFull);
  tiles_ = (uint4 *)dmalloc((u64)tile_cap_ * sizeof(uint4));
  ctl_ = (Ctl *)dmalloc(sizeof(Ctl));
  void *hc = nullptr;
  CK(cudaHostAlloc(&hc, sizeof(Ctl), cudaHostAllocDefault));
  hallocs_.push_back(hc);
  h_ctl_ = (Ctl *)hc;
  void *hdp = nullptr;
  CK(cudaHostAlloc(&hdp, 8, cudaHostAllocDefault));
  hallocs_.push_back(hdp);
  h_dpacked_ = (u64 *)hdp;
  if (opt_.algo == DYCG_ALGO_PR) {
    x_ = (float *)dmalloc((n + 1ull) * 4);
    r_ = (float *)dmalloc((n + 1ull) * 4);
    delta_ = (float *)dmalloc((n + 1ull) * 4);
    queued_ = (uint32_t *)dmalloc((n + 1ull) * 4);
    CK(cudaMemsetAsync(delta_, 0, (n + 1ull) * 4, st_));
  }
  sync_check("state");
  loaded_ = true;
}

void Engine::load_csr(uint32_t n, const uint64_t *off, const uint32_t *dst, const uint32_t *w) {
  if (loaded_) throw Error(DYCG_ESTATE, "graph already loaded");
  if (n == 0 || n >= 0x7FFFFFFFu) throw Error(DYCG_EINVAL, "vertex count out of range");
  if (!off || (!dst && off[n] != 0)) throw Error(DYCG_EINVAL, "null CSR array");
  if (off[0] != 0) throw Error(DYCG_EINVAL, "CSR offsets must start at 0");
  for (uint32_t v = 0; v < n; v++)
    if (off[v] > off[v + 1]) throw Error(DYCG_EINVAL, "CSR offsets must not decrease");
  n_ = n;
  const u64 m = off[n];
  for (u64 e = 0; e < m; e++)
    if (dst[e] >= n) throw Error(DYCG_EINVAL, "CSR neighbour id out of range");
  const bool with_w = stored_;
  u64 *d_off = nullptr;
  uint32_t *d_dst = nullptr, *d_w = nullptr, *d_w2 = nullptr;
  u64 *k1 = nullptr, *k2 = nullptr;
  CK(cudaMalloc(&d_off, (n + 1ull) * 8));
  CK(cudaMalloc(&d_dst, std::max<u64>(m, 1) * 4));
  CK(cudaMalloc(&k1, std::max<u64>(m, 1) * 8));
  CK(cudaMalloc(&k2, std::max<u64>(m, 1) * 8));
  CK(cudaMemcpyAsync(d_off, off, (n + 1ull) * 8, cudaMemcpyHostToDevice, st_));
  if (m) CK(cudaMemcpyAsync(d_dst, dst, m * 4, cudaMemcpyHostToDevice, st_));
  if (with_w) {
    CK(cudaMalloc(&d_w, std::max<u64>(m, 1) * 4));
    CK(cudaMalloc(&d_w2, std::max<u64>(m, 1) * 4));
    if (w && m) {
      CK(cudaMemcpyAsync(d_w, w, m * 4, cudaMemcpyHostToDevice, st_));
    } else {
      std::vector<uint32_t> ones(std::max<u64>(m, 1), 1u);
      CK(cudaMemcpyAsync(d_w, ones.data(), m * 4, cudaMemcpyHostToDevice, st_));
      sync_check("ones");
    }
  }
  CK(build_csr_keys(d_off, d_dst, n, k1, st_));
  size_t tb = 0;
  CK(build_sort(nullptr, tb, k1, k2, with_w ? d_w : nullptr, with_w ? d_w2 : nullptr, m, st_));
  void *temp = nullptr;
  CK(cudaMalloc(&temp, std::max<size_t>(tb, 16)));
  CK(build_sort(temp, tb, k1, k2, with_w ? d_w : nullptr, with_w ? d_w2 : nullptr, m, st_));
  sync_check("csr sort");
  cudaFree(temp);
  cudaFree(d_off);
  cudaFree(d_dst);
  // k2 / d_w2: sorted keys and weights; k1 / d_w are free for scratch
  build_from_sorted_keys(k2, with_w ? d_w2 : nullptr, m, false, 0, 1, 1, k1, d_w);
  cudaFree(k1);
  cudaFree(k2);
  if (d_w) cudaFree(d_w);
  if (d_w2) cudaFree(d_w2);
}

// Text edge list ("u v [w]" lines; empty, '#' and '%' lines skipped; the
// weight defaults to 1) -> CSR with each row's edges in file order.
TextGraph parse_text_graph(const char *path, uint32_t min_nodes, int weighted) {
  std::ifstream in(path);
  if (!in) throw Error(DYCG_EIO, std::string("cannot open graph file ") + path);
  std::vector<uint32_t> us, vs, ws;
  std::string line;
  uint64_t maxid = 0;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#' || line[0] == '%') continue;
    std::istringstream ss(line);
    uint64_t u, v, w = 1;
    if (!(ss >> u >> v)) continue;
    if (weighted && !(ss >> w)) w = 1;
    if (u >= 0x7FFFFFFFull || v >= 0x7FFFFFFFull) throw Error(DYCG_EIO, "vertex id too large");
    us.push_back((uint32_t)u);
    vs.push_back((uint32_t)v);
    ws.push_back((uint32_t)w);
    maxid = std::max(maxid, std::max(u, v));
  }
  TextGraph g;
  g.n = std::max<uint32_t>(us.empty() ? 1u : (uint32_t)(maxid + 1), min_nodes);
  g.off.assign(g.n + 1ull, 0);
  for (uint32_t u : us) g.off[u + 1]++;
  for (uint32_t v = 0; v < g.n; v++) g.off[v + 1] += g.off[v];
  g.dst.resize(us.size() + 1);
  g.w.resize(us.size() + 1);
  std::vector<uint64_t> fill(g.off.begin(), g.off.end() - 1);
  for (size_t i = 0; i < us.size(); i++) {
    const uint64_t p = fill[us[i]]++;
    g.dst[p] = vs[i];
    g.w[p] = ws[i];
  }
  g.m = us.size();
  return g;
}

void Engine::load_file(const char *path, uint32_t min_nodes, int weighted) {
  const TextGraph g = parse_text_graph(path, min_nodes, weighted);
  load_csr(g.n, g.off.data(), g.dst.data(), weighted ? g.w.data() : nullptr);
}

// Binary CSR: header "DYCGCSR1", n, m, flags; offsets[n+1] (u64); dst[m] (u32);
// w[m] (u32, flag bit 0). Mapped read-only; the arrays feed load_csr directly.
void Engine::load_binary(const char *path) {
  int fd = ::open(path, O_RDONLY);
  if (fd < 0) throw Error(DYCG_EIO, std::string("cannot open graph file ") + path);
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size < 32) {
    ::close(fd);
    throw Error(DYCG_EIO, "binary graph file too short");
  }
  void *map = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (map == MAP_FAILED) throw Error(DYCG_EIO, "cannot map binary graph file");
  const char *b = (const char *)map;
  uint64_t hdr[3];
  std::memcpy(hdr, b + 8, 24);
  const uint64_t n = hdr[0], m = hdr[1], flags = hdr[2];
  const uint64_t need = 32 + (n + 1) * 8 + m * 4 * ((flags & 1) ? 2 : 1);
  if (std::memcmp(b, "DYCGCSR1", 8) != 0 || n == 0 || n >= 0x7FFFFFFFull ||
      (uint64_t)st.st_size < need) {
    munmap(map, (size_t)st.st_size);
    throw Error(DYCG_EIO, "not a DYCGCSR1 file or truncated");
  }
  const uint64_t *off = (const uint64_t *)(b + 32);
  const uint32_t *dst = (const uint32_t *)(b + 32 + (n + 1) * 8);
  const uint32_t *w = (flags & 1) ? dst + m : nullptr;
  try {
    if (off[0] != 0 || off[n] != m) throw Error(DYCG_EIO, "inconsistent offsets");
    load_csr((uint32_t)n, off, dst, w);
  } catch (...) {
    munmap(map, (size_t)st.st_size);
    throw;
  }
  munmap(map, (size_t)st.st_size);
}

void Engine::load_rmat(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed,
                       uint32_t wlo, uint32_t whi, int symmetrize) {
  if (loaded_) throw Error(DYCG_ESTATE, "graph already loaded");
  if (scale < 1 || scale > 30 || ef == 0) throw Error(DYCG_EINVAL, "bad R-MAT size");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) throw Error(DYCG_EINVAL, "bad R-MAT probabilities");
  if (wlo == 0 || whi < wlo) throw Error(DYCG_EINVAL, "bad weight range");
  n_ = 1u << scale;
  const u64 draws = (u64)ef << scale;
  const u64 total = draws * (symmetrize ? 2 : 1);
  u64 *k1 = nullptr, *k2 = nullptr;
  uint32_t *flag = nullptr;
  u64 *pos = nullptr;
  CK(cudaMalloc(&k1, total * 8));
  CK(cudaMalloc(&k2, total * 8));
  CK(build_gen_rmat(k1, draws, seed, scale, a, b, c, symmetrize, st_));
  size_t tb = build_temp_bytes(total, false);
  void *temp = nullptr;
  CK(cudaMalloc(&temp, std::max<size_t>(tb, 16)));
  CK(build_sort(temp, tb, k1, k2, nullptr, nullptr, total, st_));
  CK(cudaMalloc(&flag, total * 4));
  CK(cudaMalloc(&pos, total * 8));
  CK(build_unique(k2, nullptr, total, 1, flag, pos, k1, nullptr, temp, tb, st_));
  u64 last_pos = 0;
  uint32_t last_flag = 0;
  CK(cudaMemcpyAsync(&last_pos, pos + total - 1, 8, cudaMemcpyDeviceToHost, st_));
  CK(cudaMemcpyAsync(&last_flag, flag + total - 1, 4, cudaMemcpyDeviceToHost, st_));
  sync_check("rmat unique");
  const u64 m = last_pos + last_flag;
  cudaFree(flag);
  cudaFree(pos);
  cudaFree(temp);
  build_from_sorted_keys(k1, nullptr, m, stored_, seed ^ 0x5745494748545321ull, wlo, whi, k2,
                         nullptr);
  cudaFree(k1);
  cudaFree(k2);
}

void Engine::load_grid(uint32_t side, uint32_t permille, uint32_t radius, uint64_t seed,
                       uint32_t wlo, uint32_t whi) {
  if (loaded_) throw Error(DYCG_ESTATE, "graph already loaded");
  if (side < 2 || (u64)side * side >= 0x7FFFFFFFull || radius == 0)
    throw Error(DYCG_EINVAL, "bad grid size");
  if (wlo == 0 || whi < wlo) throw Error(DYCG_EINVAL, "bad weight range");
  n_ = side * side;
  const u64 nshort = (u64)n_ * permille / 1000;
  const u64 total = (u64)n_ * 4 + nshort * 2;
  u64 *k1 = nullptr, *k2 = nullptr, *pos = nullptr;
  uint32_t *flag = nullptr;
  CK(cudaMalloc(&k1, total * 8));
  CK(cudaMalloc(&k2, total * 8));
  CK(build_gen_grid(k1, side, nshort, radius, seed, st_));
  size_t tb = build_temp_bytes(total, false);
  void *temp = nullptr;
  CK(cudaMalloc(&temp, std::max<size_t>(tb, 16)));
  CK(build_sort(temp, tb, k1, k2, nullptr, nullptr, total, st_));
  CK(cudaMalloc(&flag, total * 4));
  CK(cudaMalloc(&pos, total * 8));
  CK(build_unique(k2, nullptr, total, 1, flag, pos, k1, nullptr, temp, tb, st_));
  u64 last_pos = 0;
  uint32_t last_flag = 0;
  CK(cudaMemcpyAsync(&last_pos, pos + total - 1, 8, cudaMemcpyDeviceToHost, st_));
  CK(cudaMemcpyAsync(&last_flag, flag + total - 1, 4, cudaMemcpyDeviceToHost, st_));
  sync_check("grid unique");
  const u64 m = last_pos + last_flag;
  cudaFree(flag);
  cudaFree(pos);
  cudaFree(temp);
  build_from_sorted_keys(k1, nullptr, m, stored_, seed ^ 0x5745494748545321ull, wlo, whi, k2,
                         nullptr);
  cudaFree(k1);
  cudaFree(k2);
}

// ---- solve / batches -------------------------------------------------------

void Engine::init() {
  check_loaded();
  if (inited_) throw Error(DYCG_ESTATE, "engine already initialised");
  CK(cudaMemsetAsync(ctl_, 0, sizeof(Ctl), st_));
  const u64 timeout = 120ull * 1000000000ull;
  if (policy_ == DYCG_CACHE_LEARNED) policy_alloc();
  if (nq_) {
    init_queries(timeout);
    inited_ = true;
    cache_maintenance(true, nullptr);
    return;
  }
  if (opt_.algo == DYCG_ALGO_PR) {
    CK(launch_pr_init(x_, r_, queued_, q0_, n_, 1.f - opt_.alpha, ctl_, st_));
    PrLaunch L{};
    L.out = adj(out_);
    L.x = x_;
    L.r = r_;
    L.delta = delta_;
    L.queued = queued_;
    L.q0 = q0_;
    L.q1 = q1_;
    L.sources = touched_ ? touched_ : q0_;
    L.n_sources = counts_ ? counts_ + 4 : nullptr;
    L.tiles = tiles_;
    L.tile_cap = tile_cap_;
    L.ctl = ctl_;
    L.n = n_;
    L.cur = 0;
    L.phases = PR_CONVERGE;
    L.eps = opt_.epsilon;
    L.alpha = opt_.alpha;
    L.max_rounds = opt_.max_rounds;
    L.timeout_ns = timeout;
    L.num_sms = num_sms_;
    CK(launch_pr(L, st_));
    launches_ += 2;
  } else {
    CK(launch_init_state(opt_.algo, key_, n_, opt_.source, q0_, ctl_, st_));
    RepairLaunch L{};
    L.out = adj(out_);
    L.in = has_in_ ? adj(in_) : adj(out_);
    L.key = key_;
    L.mark = mark_;
    L.wtag = wtag_;
    L.aff = aff_;
    L.q0 = q0_;
    L.q1 = q1_;
    L.tiles = tiles_;
    L.tile_cap = tile_cap_;
    L.ctl = ctl_;
    L.n = n_;
    L.source = opt_.source;
    L.epoch = ++epoch_;
    L.tag_base = tag_base_;
    L.phases = PH_CLOSE;
    L.max_waves = (uint32_t)std::min<u64>(4ull * n_ + 1024, 0x7FFFFFFFull);
    L.delta = opt_.ordered_delta;
    L.q2 = q2_;
    L.timeout_ns = timeout;
    L.algo = opt_.algo;
    L.stored = stored_;
    L.num_sms = num_sms_;
    L.sched = opt_.frontier_queue;
    CK(launch_repair(L, st_));
    launches_ += 2;
  }
  CK(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
  sync_check("init");
  if (h_ctl_->err) {
    failed = true;
    throw Error(h_ctl_->err == ERR_WAVES || h_ctl_->err == ERR_BARRIER ? DYCG_ELIMIT : DYCG_ECAPACITY,
                "static solve failed on the device (error code " + std::to_string(h_ctl_->err) + ")");
  }
  tag_base_ += h_ctl_->waves + 2;
  if (opt_.algo == DYCG_ALGO_PR) {
    pr_cur_ = h_ctl_->pad[0];
    pr_count_ = h_ctl_->pad[1];
  }
  inited_ = true;
  cache_maintenance(true, nullptr);
}

void Engine::reserve_batch(size_t max_records) {
  check_loaded();
  if (max_records > 0x3FFFFFFFull) throw Error(DYCG_EINVAL, "batch too large");
  if (inited_ && nq_ && qmode_ == DYCG_QUERIES_BATCHED) {
    // multi-snapshot replay: buffers for the largest padding class, and the
    // graph of every class up to it captured now rather than on first use
    uint32_t top = 1024;
    while (top < max_records) top *= 2;
    ensure_batch(top);
    for (uint32_t c = 1024; c <= top; c *= 2) graph_for(c);
  } else {
    ensure_batch(std::max<size_t>(max_records, 1));
    // deferred deletions: hub rows' unsorted suffixes, a few slots per record
    ensure_defer(4ull * max_records);
  }
  sync_check("reserve batch");
}

void Engine::ensure_batch(size_t cnt) {
  if (cnt <= bcap_) return;
  drop_graphs();  // captured graphs hold the old buffers
  for (void *p : batch_allocs_) cudaFree(p);
  batch_allocs_.clear();
  size_t c = std::max<size_t>(cnt, 1024);
  c = std::max(c, bcap_ * 2);
  auto al = [&](size_t bytes) {
    void *p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    batch_allocs_.push_back(p);
    return p;
  };
  k_tmp_out_ = (u64 *)al(c * 8);
  k_tmp_in_ = (u64 *)al(c * 8);
  k_del_out_ = (u64 *)al(c * 8);
  k_del_in_ = (u64 *)al(c * 8);
  k_add_out_ = (u64 *)al(c * 8);
  k_add_in_ = (u64 *)al(c * 8);
  w_tmp_ = (uint32_t *)al(c * 4);
  w_add_out_ = (uint32_t *)al(c * 4);
  w_add_in_ = (uint32_t *)al(c * 4);
  uv_out_ = (uint2 *)al(c * 8);
  uv_in_ = (uint2 *)al(c * 8);
  mult_out_ = (uint32_t *)al(c * 4);
  mult_in_ = (uint32_t *)al(c * 4);
  found_out_ = (uint32_t *)al(c * 4);
  seg_out_ = (uint3 *)al(c * 12);
  seg_in_ = (uint3 *)al(c * 12);
  add_uvw_ = (uint3 *)al(c * 12);
  touched_ = (uint32_t *)al(c * 2 * 4);
  counts_ = (uint32_t *)al(64);
  reloc_.rec = (RelocRec *)al(c * sizeof(RelocRec));
  reloc_.cap = (uint32_t)c;
  {
    const u64 maxslots = std::max(out_.slots, in_.slots);
    const u64 cc = std::min<u64>(maxslots / RELOC_CHUNK + c + 1024, 0x7FFFFFFFull);
    reloc_.chunks = (uint2 *)al(cc * sizeof(uint2));
    reloc_.chunk_cap = (uint32_t)cc;
  }
  reloc_.n_reloc = counts_ + 8;
  reloc_.n_chunks = counts_ + 9;
  tombs_.pos = (u64 *)al(c * 8);
  tombs_.count = counts_ + 10;
  tombs_.cap = (uint32_t)c;
  defer_.on = true;
  defer_.rem = (uint32_t *)al(c * 4);
  defer_.row_u = (uint32_t *)al(c * 4);
  defer_.row_base = (u64 *)al(c * 8);
  defer_.packed = (u64 *)(counts_ + 12);  // 8-byte aligned slot of the counters
  defer_.cap_rows = (uint32_t)c;
  d_edges_ = (dycg_edge_dev *)al(c * 2 * sizeof(dycg_edge_dev));
  runs_.flags = (uint32_t *)al(c * 4);
  runs_.pos = (uint32_t *)al(c * 4);
  runs_.start = (uint32_t *)al(c * 4);
  runs_.valid = counts_ + 14;
  size_t a = 0, b = 0;
  CK(sort_keys(nullptr, a, k_tmp_out_, k_del_out_, (uint32_t)c, st_));
  CK(sort_pairs(nullptr, b, k_tmp_out_, k_add_out_, w_tmp_, w_add_out_, (uint32_t)c, st_));
  cub_bytes_ = std::max(std::max(a, b), unique_runs_temp_bytes((uint32_t)c));
  cub_temp_ = al(cub_bytes_);
  runs_.temp = cub_temp_;  // used between the sorts, on the same stream
  runs_.temp_bytes = cub_bytes_;
  if (h_stage_) {
    cudaFreeHost(h_stage_);
    hallocs_.erase(std::find(hallocs_.begin(), hallocs_.end(), (void *)h_stage_));
  }
  void *hs = nullptr;
  CK(cudaHostAlloc(&hs, c * 2 * sizeof(dycg_edge), cudaHostAllocDefault));
  hallocs_.push_back(hs);
  h_stage_ = (dycg_edge *)hs;
  bcap_ = c;
}

// Deletions of one adjacency direction. Rows with a long unsorted suffix are
// matched by sort-merge; that needs the gathered size on the host (one
// synchronisation), so a captured graph keeps the per-record scan.
void Engine::delete_direction(const Adj &A, const uint2 *uv, const uint32_t *mult,
                              const uint32_t *n_ptr, uint32_t nd, uint32_t *found,
                              int count_missing, bool capture) {
  if (capture) {
    CK(launch_delete_rows(A, uv, mult, n_ptr, nd, found, ctl_, count_missing, tombs_, mut_ctas_,
                          st_));
    launches_ += 2;
    return;
  }
  CK(launch_delete_prefix(A, uv, mult, n_ptr, nd, found, ctl_, count_missing, tombs_, defer_,
                          mut_ctas_, st_));
  CK(cudaMemcpyAsync(h_dpacked_, defer_.packed, 8, cudaMemcpyDeviceToHost, st_));
  sync_check("deferred deletions");
  const u64 pk = *h_dpacked_;
  const uint32_t nrows = (uint32_t)(pk >> 40);
  const u64 total = pk & ((1ull << 40) - 1);
  if (total > dbuf_cap_) ensure_defer(total);
  CK(launch_delete_suffix(A, uv, n_ptr, nd, found, ctl_, count_missing, tombs_, defer_, nrows,
                          total, dbufs_, st_));
  launches_ += 2 + (nrows ? 7 : 0);
}

// Sort buffers of the deferred deletions, for at least `slots` suffix slots.
// They grow geometrically (at least doubling), and reserve_batch sizes them
// ahead, because an allocation between a snapshot's stage events leaves the
// GPU idle for as long as the driver takes (hundreds of ms when another
// process holds the driver's locks, e.g. a monitoring query).
void Engine::ensure_defer(u64 slots) {
  if (slots <= dbuf_cap_) return;
  CK(cudaStreamSynchronize(st_));
  for (void *p : {(void *)dbufs_.k_in, (void *)dbufs_.k_out, (void *)dbufs_.v_in,
                  (void *)dbufs_.v_out, dbufs_.temp})
    cudaFree(p);
  dbufs_ = DeferBufs{};
  const u64 c = std::max<u64>({slots + slots / 2, dbuf_cap_ * 2, 1ull << 20});
  dbuf_cap_ = 0;
  CK(cudaMalloc((void **)&dbufs_.k_in, c * 8));
  CK(cudaMalloc((void **)&dbufs_.k_out, c * 8));
  CK(cudaMalloc((void **)&dbufs_.v_in, c * 4));
  CK(cudaMalloc((void **)&dbufs_.v_out, c * 4));
  dbufs_.temp_bytes = delete_sort_temp_bytes(c);
  CK(cudaMalloc(&dbufs_.temp, std::max<size_t>(dbufs_.temp_bytes, 16)));
  dbuf_cap_ = c;
}

// Device half of a snapshot on st_: counters reset, ingest, mutation and
// repair, no host synchronisation. capture: being recorded into a CUDA graph
// (no stage events, no touched-source pass).
void Engine::enqueue_snapshot(const dycg_edge_dev *d_dels, size_t nd, const dycg_edge_dev *d_adds,
                              size_t na, bool capture) {
  CK(cudaMemsetAsync(ctl_, 0, sizeof(Ctl), st_));
  CK(cudaMemsetAsync(counts_, 0, 64, st_));
  if (opt_.algo == DYCG_ALGO_PR) {
    // carried frontier length
    h_ctl_->q_count[pr_cur_] = pr_count_;
    CK(cudaMemcpyAsync(&ctl_->q_count[pr_cur_], &h_ctl_->q_count[pr_cur_], 4,
                       cudaMemcpyHostToDevice, st_));
  }
  launches_ += 2;
  // ---- ingest
  u64 *invalid = &ctl_->stat[ST_INVALID];
  size_t tb = cub_bytes_;
  if (nd) {
    CK(launch_prep_keys(d_dels, (uint32_t)nd, n_, k_tmp_out_, has_in_ ? k_tmp_in_ : nullptr,
                        nullptr, invalid, st_));
    CK(sort_keys(cub_temp_, tb, k_tmp_out_, k_del_out_, (uint32_t)nd, st_));
    CK(launch_unique_runs(k_del_out_, (uint32_t)nd, uv_out_, mult_out_, counts_ + 0,
                          (uint32_t)bcap_, &ctl_->err, runs_, st_));
    launches_ += 5;
    if (has_in_) {
      tb = cub_bytes_;
      CK(sort_keys(cub_temp_, tb, k_tmp_in_, k_del_in_, (uint32_t)nd, st_));
      CK(launch_unique_runs(k_del_in_, (uint32_t)nd, uv_in_, mult_in_, counts_ + 1,
                            (uint32_t)bcap_, &ctl_->err, runs_, st_));
      launches_ += 4;
    }
  }
  if (na) {
    tb = cub_bytes_;
    CK(launch_prep_keys(d_adds, (uint32_t)na, n_, k_tmp_out_, has_in_ ? k_tmp_in_ : nullptr,
                        w_tmp_, invalid, st_));
    CK(sort_pairs(cub_temp_, tb, k_tmp_out_, k_add_out_, w_tmp_, w_add_out_, (uint32_t)na, st_));
    CK(launch_row_segments(k_add_out_, (uint32_t)na, seg_out_, counts_ + 2, (uint32_t)bcap_,
                           &ctl_->err, runs_, st_));
    CK(launch_keys_to_uvw(k_add_out_, w_add_out_, (uint32_t)na, add_uvw_, st_));
    launches_ += 4;
    if (has_in_) {
      tb = cub_bytes_;
      CK(sort_pairs(cub_temp_, tb, k_tmp_in_, k_add_in_, w_tmp_, w_add_in_, (uint32_t)na, st_));
      CK(launch_row_segments(k_add_in_, (uint32_t)na, seg_in_, counts_ + 3, (uint32_t)bcap_,
                             &ctl_->err, runs_, st_));
      launches_ += 2;
    }
  }
  // distinct touched sources (PR amends and the touched_sources counter);
  // a captured graph would replay one epoch, so replays leave it out
  if (!capture) {
    ++touch_epoch_;
    if (nd) CK(launch_touched(k_del_out_, (uint32_t)nd, touch_, touch_epoch_, touched_, counts_ + 4,
                              ctl_, st_));
    if (na) CK(launch_touched(k_add_out_, (uint32_t)na, touch_, touch_epoch_, touched_, counts_ + 4,
                              ctl_, st_));
    launches_ += (nd ? 1 : 0) + (na ? 1 : 0);
  }
  if (!capture) CK(cudaEventRecord(ev_[1], st_));
  // the previous call's page staging (side stream) ends before this snapshot
  // reads or writes adjacency (a capture begins only after a join)
  if (!capture) join_staging();
  const u64 timeout = 60ull * 1000000000ull;
  PrLaunch PL{};
  if (opt_.algo == DYCG_ALGO_PR) {
    PL.out = adj(out_);
    PL.x = x_;
    PL.r = r_;
    PL.delta = delta_;
    PL.queued = queued_;
    PL.q0 = q0_;
    PL.q1 = q1_;
    PL.sources = touched_;
    PL.n_sources = counts_ + 4;
    PL.tiles = tiles_;
    PL.tile_cap = tile_cap_;
    PL.ctl = ctl_;
    PL.n = n_;
    PL.cur = pr_cur_;
    PL.del_uv = uv_out_;
    PL.del_found = found_out_;
    PL.n_del = counts_ + 0;
    PL.add_uvw = add_uvw_;
    PL.n_add = (uint32_t)na;
    PL.eps = opt_.epsilon;
    PL.alpha = opt_.alpha;
    PL.max_rounds = opt_.max_rounds;
    PL.timeout_ns = timeout;
    PL.num_sms = num_sms_;
    // the amend after the mutation needs each touched source's old degree
    if (nd + na) {
      CK(launch_pr_old_degree(touched_, counts_ + 4, (uint32_t)(nd + na), out_.live, delta_, st_));
      launches_++;
    }
  }
  // ---- mutation
  const Adj A_out = adj(out_);
  const Adj A_in = has_in_ ? adj(in_) : A_out;
  if (nd) {
    delete_direction(A_out, uv_out_, mult_out_, counts_ + 0, (uint32_t)nd, found_out_, 1, capture);
    if (has_in_)
      delete_direction(A_in, uv_in_, mult_in_, counts_ + 1, (uint32_t)nd, nullptr, 0, capture);
  }
  if (na) {
    CK(launch_add_rows(A_out, k_add_out_, w_add_out_, seg_out_, counts_ + 2, (uint32_t)na,
                       reloc_, ctl_, mut_ctas_, st_));
    launches_ += 3;
    if (has_in_) {
      CK(launch_add_rows(A_in, k_add_in_, w_add_in_, seg_in_, counts_ + 3, (uint32_t)na, reloc_,
                         ctl_, mut_ctas_, st_));
      launches_ += 3;
    }
  }
  if (!capture) CK(cudaEventRecord(ev_[2], st_));
  // learned admission / trace features, between mutation and repair: rows
  // that moved to new blocks in this snapshot are seen at their new pages
  if (feat_ && (policy_ == DYCG_CACHE_LEARNED || (!capture && trace_n_ < trace_cap_)))
    policy_prefetch(nd, na, capture);
  // ---- repair
  if (opt_.algo == DYCG_ALGO_PR) {
    PL.phases = (nd + na) ? (PR_AMEND | PR_CONVERGE) : PR_CONVERGE;
    CK(launch_pr(PL, st_));
    launches_++;
  } else if (nq_) {
    if (tune_) tune_repair((uint32_t)nd, (uint32_t)na, timeout);
    else repair_queries((uint32_t)nd, (uint32_t)na, timeout);
  } else {
    RepairLaunch L{};
    L.out = A_out;
    L.in = A_in;
    L.key = key_;
    L.mark = mark_;
    L.wtag = wtag_;
    L.aff = aff_;
    L.q0 = q0_;
    L.q1 = q1_;
    L.tiles = tiles_;
    L.tile_cap = tile_cap_;
    L.ctl = ctl_;
    L.del_uv = uv_out_;
    L.del_found = found_out_;
    L.n_del_ptr = counts_ + 0;
    L.add_uvw = add_uvw_;
    L.n_add = (uint32_t)na;
    L.n = n_;
    L.source = opt_.source;
    L.epoch = ++epoch_;
    L.tag_base = tag_base_;
    L.phases = (nd ? PH_DELETE : 0) | (na ? PH_INSERT : 0) | PH_CLOSE;
    L.max_waves = (uint32_t)std::min<u64>(4ull * n_ + 1024, 0x7FFFFFFFull);
    L.delta = opt_.ordered_delta;
    L.q2 = q2_;
    L.timeout_ns = timeout;
    L.algo = opt_.algo;
    L.stored = stored_;
    L.num_sms = num_sms_;
    L.sched = opt_.frontier_queue;
    CK(launch_repair(L, st_));
    launches_++;
  }
  if (!capture) CK(cudaEventRecord(ev_[3], st_));
  // a replayed snapshot keeps its cache maintenance inside the graph
  if (capture) maintenance_device();
}

void Engine::apply(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na,
                   bool device_ptrs, int mode, bool maintenance, dycg_batch_stats *stats) {
  check_loaded();
  if (!inited_) throw Error(DYCG_ESTATE, "dycg_init must run before batches");
  if (failed) throw Error(DYCG_ESTATE, "engine is in a failed state");
  if ((nd && !dels) || (na && !adds)) throw Error(DYCG_EINVAL, "null update array");
  if (nd > 0x3FFFFFFFull || na > 0x3FFFFFFFull) throw Error(DYCG_EINVAL, "batch too large");
  if (mode == 1) na = 0;
  if (mode == 2) nd = 0;
  ensure_batch(std::max<size_t>(std::max(nd, na), 1));
  const uint64_t l0 = launches_;
  CK(cudaEventRecord(ev_[0], st_));
  const dycg_edge_dev *d_dels = (const dycg_edge_dev *)dels;
  const dycg_edge_dev *d_adds = (const dycg_edge_dev *)adds;
  if (!device_ptrs) {
    if (nd) std::memcpy(h_stage_, dels, nd * sizeof(dycg_edge));
    if (na) std::memcpy(h_stage_ + nd, adds, na * sizeof(dycg_edge));
    if (nd + na)
      CK(cudaMemcpyAsync(d_edges_, h_stage_, (nd + na) * sizeof(dycg_edge),
                         cudaMemcpyHostToDevice, st_));
    d_dels = d_edges_;
    d_adds = d_edges_ + nd;
  }
  enqueue_snapshot(d_dels, nd, d_adds, na, false);
  CK(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
  if (nq_) {
    if (qmode_ == DYCG_QUERIES_PER_QUERY)
      CK(cudaMemcpyAsync(h_qctl_, qctl_, (u64)nq_ * sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
    CK(cudaMemcpyAsync(h_seq_, seq_, 8, cudaMemcpyDeviceToHost, st_));
  }
  sync_check("batch");
  Ctl c = *h_ctl_;
  if (nq_ && qmode_ == DYCG_QUERIES_PER_QUERY) {
    // mutation counters are in ctl_, each query's repair counters in its own block
    for (uint32_t q = 0; q < nq_; q++) {
      const Ctl &r = h_qctl_[q];
      if (!c.err) c.err = r.err;
      for (int i : {ST_LINK_BYTES, ST_HBM_ADJ_BYTES, ST_EXPANDED, ST_SCANNED, ST_IMPROVED,
                    ST_AFFECTED})
        c.stat[i] += r.stat[i];
      c.waves += r.waves;
    }
  }
  if (nq_ && h_seq_[1] > 0xF0000000u) {
    // wave tags are about to wrap: clear the tag array and restart the count
    CK(cudaMemsetAsync(wtag_, 0, (n_ + 1ull) * 4, st_));
    h_seq_[1] = 1;
    CK(cudaMemcpyAsync(seq_ + 1, h_seq_ + 1, 4, cudaMemcpyHostToDevice, st_));
    sync_check("tag reset");
  }
  if (c.err) {
    failed = true;
    const int code = (c.err == ERR_WAVES || c.err == ERR_BARRIER) ? DYCG_ELIMIT : DYCG_ECAPACITY;
    throw Error(code, "batch failed on the device (error code " + std::to_string(c.err) + ")");
  }
  tag_base_ += c.waves + 2;
  if (opt_.algo == DYCG_ALGO_PR) {
    pr_cur_ = c.pad[0];
    pr_count_ = c.pad[1];
  }
  float ms[4] = {0, 0, 0, 0};
  cudaEventElapsedTime(&ms[0], ev_[0], ev_[1]);
  cudaEventElapsedTime(&ms[1], ev_[1], ev_[2]);
  cudaEventElapsedTime(&ms[2], ev_[2], ev_[3]);
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->deletions = nd;
    stats->insertions = na;
    stats->missing_deletes = c.stat[ST_MISSING];
    stats->invalid_updates = c.stat[ST_INVALID];
    stats->touched_sources = c.stat[ST_TOUCHED];
    stats->relocated_rows = c.stat[ST_RELOCATED];
    stats->affected = c.stat[ST_AFFECTED];
    stats->expanded = c.stat[ST_EXPANDED];
    stats->edges_scanned = c.stat[ST_SCANNED];
    stats->improvements = c.stat[ST_IMPROVED];
    stats->waves = c.waves;
    stats->link_bytes = c.stat[ST_LINK_BYTES] + c.stat[ST_MUT_LINK_BYTES];
    stats->hbm_adj_bytes = c.stat[ST_HBM_ADJ_BYTES] + c.stat[ST_MUT_HBM_BYTES];
    stats->mutate_link_bytes = c.stat[ST_MUT_LINK_BYTES];
    stats->mutate_hbm_bytes = c.stat[ST_MUT_HBM_BYTES];
    stats->ms_ingest = ms[0];
    stats->ms_mutate = ms[1];
    stats->ms_repair = ms[2];
    if (prefetched_) {  // the learned admission ran inside the repair stage's events
      float pm = 0;
      cudaEventElapsedTime(&pm, pev_[0], pev_[1]);
      stats->ms_repair -= pm;
    }
  }
  if (maintenance) cache_maintenance(false, stats);
  if (stats) {
    stats->kernel_launches = launches_ - l0;
    float tot = 0;
    cudaEventElapsedTime(&tot, ev_[0], maintenance && cache_slots_ ? ev_[5] : ev_[3]);
    stats->ms_total = tot;
    // repair kernels' vertex-state bytes (algorithmic): per expanded row its
    // 16-byte descriptor and 8-byte key, per scanned slot the neighbour's
    // 8-byte key, per improvement 8 B key atomic + 4 B tag + 4 B queue slot
    if (nq_ && qmode_ == DYCG_QUERIES_BATCHED) {
      // batched: the kernel counts 8 B per (edge, active query) key access
      stats->state_bytes = c.stat[ST_STATE_BYTES] + stats->expanded * 16 + stats->improvements * 16;
      fill_phases(stats, c);
    } else {
      stats->state_bytes = stats->expanded * 24 + stats->edges_scanned * 8 + stats->improvements * 16;
      if (!nq_ && opt_.algo != DYCG_ALGO_PR) fill_phases(stats, c);
    }
  }
}

// Phase times of a repair from the kernel's own timer stamps (single-source
// or batched; phases a launch skipped have no stamp and count zero).
static void fill_phases(dycg_batch_stats *s, const Ctl &c) {
  const u64 t[4] = {c.tphase[0], c.tphase[1], c.tphase[2], c.tphase[3]};
  double *out[4] = {&s->ms_phase_invalidate, &s->ms_phase_pull, &s->ms_phase_seed,
                    &s->ms_phase_closure};
  u64 prev = c.stat[ST_T_START];
  for (int i = 0; i < 4; i++) {
    *out[i] = 0;
    if (t[i] && prev && t[i] >= prev) {
      *out[i] = (t[i] - prev) * 1e-6;
      prev = t[i];
    }
  }
}

// ---- many-query forms -------------------------------------------------------

void Engine::set_queries(const uint32_t *sources, uint32_t count, uint32_t mode) {
  check_loaded();
  if (inited_) throw Error(DYCG_ESTATE, "queries must be set before dycg_init");
  if (nq_) throw Error(DYCG_ESTATE, "queries already set");
  if (opt_.algo != DYCG_ALGO_SSSP && opt_.algo != DYCG_ALGO_BFS)
    throw Error(DYCG_EINVAL, "many-query forms support SSSP and BFS");
  if (count == 0 || count > DYCG_MAX_QUERIES) throw Error(DYCG_EINVAL, "query count out of range");
  if (mode != DYCG_QUERIES_BATCHED && mode != DYCG_QUERIES_PER_QUERY)
    throw Error(DYCG_EINVAL, "unknown query mode");
  if (opt_.ordered_delta && mode == DYCG_QUERIES_BATCHED)
    throw Error(DYCG_EINVAL, "the batched form runs the unordered closure (ordered_delta 0)");
  for (uint32_t q = 0; q < count; q++)
    if (sources[q] >= n_) throw Error(DYCG_EINVAL, "query source out of range");
  sources_.assign(sources, sources + count);
  const u64 n = n_;
  if (mode == DYCG_QUERIES_BATCHED) {
    uint32_t nb = 1;
    while (nb * 32 < count) nb *= 2;
    const uint32_t Q = nb * 32;
    std::vector<uint32_t> padded(Q, INF32);
    std::copy(sources, sources + count, padded.begin());
    d_sources_ = (uint32_t *)dmalloc((u64)Q * 4);
    CK(cudaMemcpyAsync(d_sources_, padded.data(), (u64)Q * 4, cudaMemcpyHostToDevice, st_));
    qkey_ = (u64 *)dmalloc(n * Q * 8);
    uint32_t **masks[6] = {&affm_, &inew_[0], &inew_[1], &nmask_[0], &nmask_[1], &cmask_};
    for (uint32_t **m : masks) {
      *m = (uint32_t *)dmalloc(n * nb * 4);
      CK(cudaMemsetAsync(*m, 0, n * nb * 4, st_));
    }
    // tiles of one wave: at most one per MULTI_MIN_TILE slots plus one per row
    const u64 maxslots = std::max(out_.slots, in_.slots);
    mtile_cap_ = (uint32_t)std::min<u64>(maxslots / MULTI_MIN_TILE + n + 4096, 0x7FFFFFFFull);
    mtiles_ = (uint4 *)dmalloc((u64)mtile_cap_ * sizeof(uint4));
    // asynchronous worklist: one item per vertex at most, plus up to 2^20
    // tile items, plus the positions the waiting warps have claimed
    aring_cap_ = (uint32_t)std::min<u64>(n + (1ull << 20) + 65536, 0xFFFFFFFFull);
    aring_ = (u64 *)dmalloc((u64)aring_cap_ * 8);
    CK(cudaMemsetAsync(aring_, 0xFF, (u64)aring_cap_ * 8, st_));
    ainq_ = (uint32_t *)dmalloc(n * 4);
    CK(cudaMemsetAsync(ainq_, 0, n * 4, st_));
    apool_cap_ = 65535;
    apool_ = (uint32_t *)dmalloc((u64)apool_cap_ * nb * 4);
    qnb_ = nb;
    qbytes_ = (u64)Q * 4 + n * Q * 8 + 6 * n * nb * 4 + (u64)mtile_cap_ * sizeof(uint4) +
              (u64)aring_cap_ * 8 + n * 4 + (u64)apool_cap_ * nb * 4;
  } else {
    d_sources_ = (uint32_t *)dmalloc((u64)count * 4);
    CK(cudaMemcpyAsync(d_sources_, sources, (u64)count * 4, cudaMemcpyHostToDevice, st_));
    qkey_ = (u64 *)dmalloc(n * count * 8);
    qctl_ = (Ctl *)dmalloc((u64)count * sizeof(Ctl));
    void *hq = nullptr;
    CK(cudaHostAlloc(&hq, (u64)count * sizeof(Ctl), cudaHostAllocDefault));
    hallocs_.push_back(hq);
    h_qctl_ = (Ctl *)hq;
    qbytes_ = (u64)count * 4 + n * count * 8 + (u64)count * sizeof(Ctl);
  }
  seq_ = (uint32_t *)dmalloc(8);
  void *hs = nullptr;
  CK(cudaHostAlloc(&hs, 8, cudaHostAllocDefault));
  hallocs_.push_back(hs);
  h_seq_ = (uint32_t *)hs;
  h_seq_[0] = 1;  // epoch (mark_ starts at 0)
  h_seq_[1] = 1;  // next wave tag (wtag_ starts at 0)
  CK(cudaMemcpyAsync(seq_, h_seq_, 8, cudaMemcpyHostToDevice, st_));
  qmode_ = mode;
  nq_ = count;
  sync_check("queries");
}

void Engine::set_query_mapping(uint32_t qratio, uint32_t heavy, uint32_t tile) {
  if (heavy == 0) throw Error(DYCG_EINVAL, "heavy must be >= 1");
  if (tile < MULTI_MIN_TILE) throw Error(DYCG_EINVAL, "tile must be >= 1024 slots");
  qratio_ = pull_qratio_ = qratio;
  heavy_ = heavy;
  tile_ = tile;
  drop_graphs();  // captured graphs hold the old mapping
}

void Engine::set_query_queue(uint32_t scheme) {
  if (scheme > (DYCG_QUEUE_CLAIMED | DYCG_QUEUE_RANGES | DYCG_QUEUE_ASYNC))
    throw Error(DYCG_EINVAL, "unknown frontier-queue scheme");
  sched_ = scheme;
  drop_graphs();  // captured graphs hold the old scheme
}

MultiLaunch Engine::multi_launch(uint32_t phases, uint32_t n_add, u64 timeout) {
  MultiLaunch L{};
  L.out = adj(out_);
  L.in = has_in_ ? adj(in_) : L.out;
  L.key = qkey_;
  L.affm = affm_;
  L.inew0 = inew_[0];
  L.inew1 = inew_[1];
  L.nmask0 = nmask_[0];
  L.nmask1 = nmask_[1];
  L.cmask = cmask_;
  L.mark = mark_;
  L.wtag = wtag_;
  L.aff = aff_;
  L.q0 = q0_;
  L.q1 = q1_;
  L.tiles = mtiles_;
  L.tile_cap = mtile_cap_;
  L.ctl = ctl_;
  L.seq = seq_;
  L.del_uv = uv_out_;
  L.del_found = found_out_;
  L.n_del_ptr = counts_;
  L.add_uvw = add_uvw_;
  L.n_add = n_add;
  L.n = n_;
  L.nb = qnb_;
  L.phases = phases;
  L.max_waves = (uint32_t)std::min<u64>(4ull * n_ + 1024, 0x7FFFFFFFull);
  L.qratio = qratio_;
  L.pull_qratio = pull_qratio_;
  L.heavy = heavy_;
  L.tile = tile_;
  L.sched = sched_;
  L.ring = aring_;
  L.ring_cap = aring_cap_;
  L.inq = ainq_;
  L.pool = apool_;
  L.pool_cap = apool_cap_;
  L.timeout_ns = timeout;
  L.algo = opt_.algo;
  L.stored = stored_;
  L.num_sms = num_sms_;
  return L;
}

// Single-source repair launch of query q (the per-query form).
static RepairLaunch query_launch(const Adj &out, const Adj &in, u64 *key, uint32_t source) {
  RepairLaunch L{};
  L.out = out;
  L.in = in;
  L.key = key;
  L.source = source;
  return L;
}

// Static solve of every query.
void Engine::init_queries(u64 timeout) {
  if (qmode_ == DYCG_QUERIES_BATCHED) {
    CK(launch_multi_init(qkey_, n_, qnb_, d_sources_, nmask_[0], q0_, wtag_, seq_, ctl_, sched_,
                         st_));
    CK(launch_multi(multi_launch(PH_CLOSE, 0, timeout), st_));
    launches_ += 3;
    CK(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
    sync_check("init queries");
    if (h_ctl_->err) {
      failed = true;
      throw Error(h_ctl_->err == ERR_WAVES || h_ctl_->err == ERR_BARRIER ? DYCG_ELIMIT : DYCG_ECAPACITY,
                  "batched static solve failed on the device (error code " +
                      std::to_string(h_ctl_->err) + ")");
    }
    return;
  }
  CK(cudaMemsetAsync(qctl_, 0, (u64)nq_ * sizeof(Ctl), st_));
  const Adj A_out = adj(out_);
  const Adj A_in = has_in_ ? adj(in_) : A_out;
  for (uint32_t q = 0; q < nq_; q++) {
    u64 *key = qkey_ + (u64)q * n_;
    CK(launch_init_state(opt_.algo, key, n_, sources_[q], q0_, qctl_ + q, st_));
    RepairLaunch L = query_launch(A_out, A_in, key, sources_[q]);
    L.mark = mark_;
    L.wtag = wtag_;
    L.aff = aff_;
    L.q0 = q0_;
    L.q1 = q1_;
    L.tiles = tiles_;
    L.tile_cap = tile_cap_;
    L.ctl = qctl_ + q;
    L.n = n_;
    L.epoch = ++epoch_;
    L.phases = PH_CLOSE;
    L.max_waves = (uint32_t)std::min<u64>(4ull * n_ + 1024, 0x7FFFFFFFull);
    L.delta = opt_.ordered_delta;
    L.q2 = q2_;
    L.tag_dev = seq_ + 1;
    L.timeout_ns = timeout;
    L.algo = opt_.algo;
    L.stored = stored_;
    L.num_sms = num_sms_;
    L.sched = opt_.frontier_queue;
    CK(launch_repair(L, st_));
    launches_ += 2;
  }
  CK(cudaMemcpyAsync(h_qctl_, qctl_, (u64)nq_ * sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
  sync_check("init queries");
  for (uint32_t q = 0; q < nq_; q++)
    if (h_qctl_[q].err) {
      failed = true;
      throw Error(h_qctl_[q].err == ERR_WAVES || h_qctl_[q].err == ERR_BARRIER ? DYCG_ELIMIT
                                                                               : DYCG_ECAPACITY,
                  "static solve of query " + std::to_string(q) + " failed (error code " +
                      std::to_string(h_qctl_[q].err) + ")");
    }
}

// Repair of every query after the snapshot's mutation (asynchronous).
void Engine::repair_queries(uint32_t nd, uint32_t na, u64 timeout) {
  const uint32_t phases = (nd ? PH_DELETE : 0) | (na ? PH_INSERT : 0) | PH_CLOSE;
  if (qmode_ == DYCG_QUERIES_BATCHED) {
    CK(launch_multi(multi_launch(phases, na, timeout), st_));
    launches_++;
    return;
  }
  CK(cudaMemsetAsync(qctl_, 0, (u64)nq_ * sizeof(Ctl), st_));
  launches_++;
  const Adj A_out = adj(out_);
  const Adj A_in = has_in_ ? adj(in_) : A_out;
  for (uint32_t q = 0; q < nq_; q++) {
    RepairLaunch L = query_launch(A_out, A_in, qkey_ + (u64)q * n_, sources_[q]);
    L.mark = mark_;
    L.wtag = wtag_;
    L.aff = aff_;
    L.q0 = q0_;
    L.q1 = q1_;
    L.tiles = tiles_;
    L.tile_cap = tile_cap_;
    L.ctl = qctl_ + q;
    L.del_uv = uv_out_;
    L.del_found = found_out_;
    L.n_del_ptr = counts_;
    L.add_uvw = add_uvw_;
    L.n_add = na;
    L.n = n_;
    L.epoch = ++epoch_;
    L.phases = phases;
    L.max_waves = (uint32_t)std::min<u64>(4ull * n_ + 1024, 0x7FFFFFFFull);
    L.delta = opt_.ordered_delta;
    L.q2 = q2_;
    L.tag_dev = seq_ + 1;
    L.timeout_ns = timeout;
    L.algo = opt_.algo;
    L.stored = stored_;
    L.num_sms = num_sms_;
    L.sched = opt_.frontier_queue;
    CK(launch_repair(L, st_));
    launches_++;
  }
}

void Engine::gather_query(uint32_t q, uint32_t *values, uint32_t *parents) {
  check_loaded();
  if (!nq_) throw Error(DYCG_ESTATE, "no queries set");
  if (q >= nq_) throw Error(DYCG_EINVAL, "query index out of range");
  // q0_/q1_ (n+1 entries each) are idle between calls: use them as staging
  if (qmode_ == DYCG_QUERIES_BATCHED)
    CK(launch_multi_gather(qkey_, n_, qnb_ * 32, q, q0_, q1_, st_));
  else
    CK(launch_multi_gather(qkey_ + (u64)q * n_, n_, 0, 0, q0_, q1_, st_));
  if (values) CK(cudaMemcpyAsync(values, q0_, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  if (parents) CK(cudaMemcpyAsync(parents, q1_, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  sync_check("gather query");
}

// ---- mapping autotuner and multi-snapshot replay ------------------------------

// Repair of the current snapshot under every candidate mapping, each from the
// same saved state (keys, page hotness, counters); keeps the fastest mapping
// and ends with that mapping's run, so the engine state and the stage events
// describe one ordinary repair.
void Engine::tune_repair(uint32_t nd, uint32_t na, u64 timeout) {
  if (qmode_ != DYCG_QUERIES_BATCHED) {
    repair_queries(nd, na, timeout);
    return;
  }
  const uint32_t phases = (nd ? PH_DELETE : 0) | (na ? PH_INSERT : 0) | PH_CLOSE;
  const u64 kbytes = (u64)n_ * qnb_ * 32 * 8, hbytes = (u64)npages_ * 4;
  struct Scratch {
    void *p[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t a = nullptr, b = nullptr;
    ~Scratch() {
      for (void *x : p) cudaFree(x);
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } sc;
  CK(cudaMalloc(&sc.p[0], kbytes));
  CK(cudaMalloc(&sc.p[1], std::max<u64>(hbytes, 4)));
  CK(cudaMalloc(&sc.p[2], sizeof(Ctl)));
  CK(cudaEventCreate(&sc.a));
  CK(cudaEventCreate(&sc.b));
  CK(cudaMemcpyAsync(sc.p[0], qkey_, kbytes, cudaMemcpyDeviceToDevice, st_));
  CK(cudaMemcpyAsync(sc.p[1], page_hits_, hbytes, cudaMemcpyDeviceToDevice, st_));
  CK(cudaMemcpyAsync(sc.p[2], ctl_, sizeof(Ctl), cudaMemcpyDeviceToDevice, st_));
  auto restore = [&]() {
    CK(cudaMemcpyAsync(qkey_, sc.p[0], kbytes, cudaMemcpyDeviceToDevice, st_));
    CK(cudaMemcpyAsync(page_hits_, sc.p[1], hbytes, cudaMemcpyDeviceToDevice, st_));
    CK(cudaMemcpyAsync(ctl_, sc.p[2], sizeof(Ctl), cudaMemcpyDeviceToDevice, st_));
  };
  static const uint32_t kRatio[] = {2, 4, 8, 1u << 20};
  static const uint32_t kHeavy[] = {4, 8, 16, 64, 256};
  static const uint32_t kPull[] = {0, 1, 2, 8};
  static const uint32_t kTile[] = {1024, 4096, 16384};
  tried_.clear();
  const uint32_t tile0 = tile_, sched0 = sched_;
  dycg_query_mapping best{qratio_, heavy_, tile_, pull_qratio_, sched_, 1e30f};
  auto trial = [&](uint32_t r, uint32_t h, uint32_t pr, uint32_t t, uint32_t q) {
    if (!tried_.empty()) restore();
    qratio_ = r;
    heavy_ = h;
    pull_qratio_ = pr;
    tile_ = t;
    sched_ = q;
    CK(cudaEventRecord(sc.a, st_));
    CK(launch_multi(multi_launch(phases, na, timeout), st_));
    CK(cudaEventRecord(sc.b, st_));
    CK(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
    sync_check("tune");
    if (h_ctl_->err) {
      failed = true;
      throw Error(DYCG_ELIMIT, "mapping trial failed on the device (error code " +
                                   std::to_string(h_ctl_->err) + ")");
    }
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, sc.a, sc.b));
    tried_.push_back({r, h, t, pr, q, ms});
    if (ms < best.repair_ms) best = tried_.back();
    launches_++;
  };
  // coordinate search: (qratio, heavy) with the pull phase on the same rule,
  // then the pull phase's own ratio, then the slots per query-lane tile, then
  // the frontier-queue scheme
  for (uint32_t r : kRatio)
    for (uint32_t h : kHeavy) trial(r, h, r, tile0, sched0);
  const dycg_query_mapping first = best;
  for (uint32_t pr : kPull)
    if (pr != first.qratio) trial(first.qratio, first.heavy, pr, tile0, sched0);
  const dycg_query_mapping second = best;
  for (uint32_t t : kTile)
    if (t != second.tile) trial(second.qratio, second.heavy, second.pull_qratio, t, sched0);
  const dycg_query_mapping third = best;
  for (uint32_t q : {DYCG_QUEUE_STATIC, DYCG_QUEUE_CLAIMED, DYCG_QUEUE_RANGES,
                     DYCG_QUEUE_CLAIMED | DYCG_QUEUE_RANGES, DYCG_QUEUE_ASYNC,
                     DYCG_QUEUE_ASYNC | DYCG_QUEUE_CLAIMED})
    if (q != third.queue) trial(third.qratio, third.heavy, third.pull_qratio, third.tile, q);
  restore();
  qratio_ = best.qratio;
  heavy_ = best.heavy;
  pull_qratio_ = best.pull_qratio;
  tile_ = best.tile;
  sched_ = best.queue;
  drop_graphs();
  CK(cudaEventRecord(ev_[2], st_));  // the stage boundary of the kept run
  CK(launch_multi(multi_launch(phases, na, timeout), st_));
  launches_++;
  sync_check("tune final");  // scratch is released on return
}

void Engine::tune(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na,
                  dycg_query_mapping *tried, uint32_t cap, uint32_t *n_tried,
                  dycg_batch_stats *stats) {
  if (!nq_ || qmode_ != DYCG_QUERIES_BATCHED)
    throw Error(DYCG_ESTATE, "mapping tuning needs the batched many-query form");
  tune_ = true;
  try {
    apply(dels, nd, adds, na, false, 0, true, stats);
  } catch (...) {
    tune_ = false;
    throw;
  }
  tune_ = false;
  if (n_tried) *n_tried = (uint32_t)tried_.size();
  for (uint32_t i = 0; tried && i < cap && i < tried_.size(); i++) tried[i] = tried_[i];
}

void Engine::drop_graphs() {
  for (auto &g : graphs_) cudaGraphExecDestroy(g.second.exec);
  graphs_.clear();
}

// Graph of one snapshot of padded size cls (records at d_edges_: deletions
// [0, cls), insertions [cls, 2 cls)), captured on first use.
const Engine::SnapshotGraph &Engine::graph_for(uint32_t cls) {
  auto it = graphs_.find(cls);
  if (it != graphs_.end()) return it->second;
  join_staging();
  cudaGraph_t g = nullptr;
  const uint64_t l0 = launches_;
  CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_snapshot(d_edges_, cls, d_edges_ + cls, cls, true);
  } catch (...) {
    cudaStreamEndCapture(st_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  CK(cudaStreamEndCapture(st_, &g));
  SnapshotGraph sg{nullptr, launches_ - l0};
  const cudaError_t e = cudaGraphInstantiate(&sg.exec, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  launches_ = l0;
  return graphs_.emplace(cls, sg).first->second;
}

void Engine::apply_batches(const dycg_edge *dels, const uint64_t *nd, const dycg_edge *adds,
                           const uint64_t *na, uint32_t count, bool device_ptrs,
                           dycg_batch_stats *stats) {
  check_loaded();
  if (!inited_) throw Error(DYCG_ESTATE, "dycg_init must run before batches");
  if (failed) throw Error(DYCG_ESTATE, "engine is in a failed state");
  if (count && (!nd || !na)) throw Error(DYCG_EINVAL, "null count array");
  u64 td = 0, ta = 0, mx = 1;
  for (uint32_t i = 0; i < count; i++) {
    if (nd[i] > 0x3FFFFFFFull || na[i] > 0x3FFFFFFFull) throw Error(DYCG_EINVAL, "batch too large");
    td += nd[i];
    ta += na[i];
    mx = std::max<u64>(mx, std::max(nd[i], na[i]));
  }
  if ((td && !dels) || (ta && !adds)) throw Error(DYCG_EINVAL, "null update array");
  // trace recording (and the snapshots whose page reads still complete the
  // traced snapshots' targets) needs the host between snapshots
  const bool tracing =
      trace_n_ < trace_cap_ || (trace_cap_ && trace_post_ + 1 < (uint32_t)POLICY_HORIZON);
  if (!(nq_ && qmode_ == DYCG_QUERIES_BATCHED) || tracing) {
    // other forms and trace recording: one ordinary apply per snapshot
    u64 od = 0, oa = 0;
    for (uint32_t i = 0; i < count; i++) {
      apply(dels + od, nd[i], adds + oa, na[i], device_ptrs, 0, true, stats ? stats + i : nullptr);
      od += nd[i];
      oa += na[i];
    }
    return;
  }
  auto cls_of = [](u64 x) {
    uint32_t c = 1024;
    while (c < x) c *= 2;
    return c;
  };
  ensure_batch(cls_of(mx));
  // records on the device: the caller's, or one staged copy of all snapshots
  const dycg_edge_dev *d_dels = (const dycg_edge_dev *)dels, *d_adds = (const dycg_edge_dev *)adds;
  if (!device_ptrs && td + ta) {
    const u64 bytes = (td + ta) * sizeof(dycg_edge);
    if (bytes > hrec_bytes_) {
      if (h_rec_) cudaFreeHost(h_rec_);
      if (d_rec_) cudaFree(d_rec_);
      h_rec_ = nullptr;
      d_rec_ = nullptr;
      hrec_bytes_ = 0;
      CK(cudaHostAlloc(&h_rec_, bytes, cudaHostAllocDefault));
      CK(cudaMalloc(&d_rec_, bytes));
      hrec_bytes_ = bytes;
    }
    if (td) std::memcpy(h_rec_, dels, td * sizeof(dycg_edge));
    if (ta) std::memcpy((char *)h_rec_ + td * sizeof(dycg_edge), adds, ta * sizeof(dycg_edge));
    CK(cudaMemcpyAsync(d_rec_, h_rec_, bytes, cudaMemcpyHostToDevice, st_));
    d_dels = (const dycg_edge_dev *)d_rec_;
    d_adds = d_dels + td;
  }
  if (count > bctl_cap_) {
    if (h_bctl_) cudaFreeHost(h_bctl_);
    h_bctl_ = nullptr;
    bctl_cap_ = 0;
    CK(cudaHostAlloc((void **)&h_bctl_, (u64)count * sizeof(Ctl), cudaHostAllocDefault));
    bctl_cap_ = count;
  }
  while (bev_.size() < 2 * (size_t)count) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    bev_.push_back(e);
  }
  std::vector<uint32_t> cls(count);
  u64 od = 0, oa = 0;
  for (uint32_t i = 0; i < count; i++) {
    cls[i] = cls_of(std::max<u64>(std::max(nd[i], na[i]), 1));
    const SnapshotGraph &g = graph_for(cls[i]);
    // padding records carry out-of-range ids: ingest drops them
    CK(cudaMemsetAsync(d_edges_, 0xFF, 2ull * cls[i] * sizeof(dycg_edge), st_));
    if (nd[i])
      CK(cudaMemcpyAsync(d_edges_, d_dels + od, nd[i] * sizeof(dycg_edge),
                         cudaMemcpyDeviceToDevice, st_));
    if (na[i])
      CK(cudaMemcpyAsync(d_edges_ + cls[i], d_adds + oa, na[i] * sizeof(dycg_edge),
                         cudaMemcpyDeviceToDevice, st_));
    CK(cudaEventRecord(bev_[2 * i], st_));
    CK(cudaGraphLaunch(g.exec, st_));
    CK(cudaEventRecord(bev_[2 * i + 1], st_));
    CK(cudaMemcpyAsync(h_bctl_ + i, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, st_));
    launches_ += g.kernels;
    od += nd[i];
    oa += na[i];
  }
  CK(cudaMemcpyAsync(h_seq_, seq_, 8, cudaMemcpyDeviceToHost, st_));
  sync_check("batches");
  for (uint32_t i = 0; i < count; i++)
    if (h_bctl_[i].err) {
      failed = true;
      const uint32_t er = h_bctl_[i].err;
      throw Error(er == ERR_WAVES || er == ERR_BARRIER ? DYCG_ELIMIT : DYCG_ECAPACITY,
                  "snapshot " + std::to_string(i) + " failed on the device (error code " +
                      std::to_string(er) + ")");
    }
  if (h_seq_[1] > 0xF0000000u) {
    CK(cudaMemsetAsync(wtag_, 0, (n_ + 1ull) * 4, st_));
    h_seq_[1] = 1;
    CK(cudaMemcpyAsync(seq_ + 1, h_seq_ + 1, 4, cudaMemcpyHostToDevice, st_));
    sync_check("tag reset");
  }
  if (stats) {
    for (uint32_t i = 0; i < count; i++) {
      const Ctl &c = h_bctl_[i];
      dycg_batch_stats *s = stats + i;
      std::memset(s, 0, sizeof(*s));
      s->deletions = nd[i];
      s->insertions = na[i];
      s->missing_deletes = c.stat[ST_MISSING];
      // padding records count as invalid in the device counter
      s->invalid_updates = c.stat[ST_INVALID] - (2ull * cls[i] - nd[i] - na[i]);
      s->relocated_rows = c.stat[ST_RELOCATED];
      s->affected = c.stat[ST_AFFECTED];
      s->expanded = c.stat[ST_EXPANDED];
      s->edges_scanned = c.stat[ST_SCANNED];
      s->improvements = c.stat[ST_IMPROVED];
      s->waves = c.waves;
      s->link_bytes = c.stat[ST_LINK_BYTES] + c.stat[ST_MUT_LINK_BYTES];
      s->hbm_adj_bytes = c.stat[ST_HBM_ADJ_BYTES] + c.stat[ST_MUT_HBM_BYTES];
      s->mutate_link_bytes = c.stat[ST_MUT_LINK_BYTES];
      s->mutate_hbm_bytes = c.stat[ST_MUT_HBM_BYTES];
      s->state_bytes = c.stat[ST_STATE_BYTES] + s->expanded * 16 + s->improvements * 16;
      s->cache_pages_loaded = c.stat[ST_PAGES_LOADED];
      s->cache_pages_evicted = c.stat[ST_PAGES_EVICTED];
      {
        const u64 page_bytes = (4ull << page_shift_) * out_.stride;
        s->link_bytes += c.stat[ST_PAGES_LOADED] * page_bytes;
        s->hbm_adj_bytes += c.stat[ST_PAGES_LOADED] * page_bytes;
      }
      s->kernel_launches = graphs_.count(cls[i]) ? graphs_[cls[i]].kernels : 0;
      float ms = 0;
      cudaEventElapsedTime(&ms, bev_[2 * i], bev_[2 * i + 1]);
      s->ms_total = ms;
      // the repair kernel's own start/end stamps (no stage events in a graph)
      if (c.stat[ST_T_END] > c.stat[ST_T_START] && c.stat[ST_T_START])
        s->ms_repair = (c.stat[ST_T_END] - c.stat[ST_T_START]) * 1e-6;
      fill_phases(s, c);
    }
  }
}

// ---- learned cache admission policy -------------------------------------------

void Engine::policy_alloc() {
  check_loaded();
  if (feat_) return;
  const u64 np = npages_;
  feat_ = dmalloc(np * POLICY_F * 2);
  hist_ = (float *)dmalloc(np * 4 * 4);
  age_ = (uint8_t *)dmalloc(np);
  prows_ = (uint32_t *)dmalloc(np * 4);
  pmax_ = (uint32_t *)dmalloc(np * 4);
  pdelta_ = (uint32_t *)dmalloc(np * 4);
  pperiod_ = (uint32_t *)dmalloc(8);
  {
    const uint32_t per[2] = {0, 8};
    CK(cudaMemcpyAsync(pperiod_, per, 8, cudaMemcpyHostToDevice, st_));
  }
  CK(cudaMemsetAsync(hist_, 0, np * 16, st_));
  CK(cudaMemsetAsync(age_, 0xFF, np, st_));
  params_ = (float *)dmalloc(POLICY_PARAMS * 4);
  grad_ = (float *)dmalloc(POLICY_PARAMS * 4);
  adam_m_ = (float *)dmalloc(POLICY_PARAMS * 4);
  adam_v_ = (float *)dmalloc(POLICY_PARAMS * 4);
  ploss_ = (float *)dmalloc(16);
  CK(cudaMemsetAsync(grad_, 0, POLICY_PARAMS * 4, st_));
  CK(cudaMemsetAsync(adam_m_, 0, POLICY_PARAMS * 4, st_));
  CK(cudaMemsetAsync(adam_v_, 0, POLICY_PARAMS * 4, st_));
  // Glorot-uniform weights from a fixed seed, zero biases
  std::vector<float> p(POLICY_PARAMS, 0.f);
  auto fill = [&](int off, int fan_in, int fan_out, u64 tag) {
    const float a = std::sqrt(6.f / (fan_in + fan_out));
    for (int i = 0; i < fan_in * fan_out; i++) {
      const double u = (double)(mix64(tag ^ mix64((u64)i + 1)) >> 11) / 9007199254740992.0;
      p[off + i] = (float)((2.0 * u - 1.0) * a);
    }
  };
  const int F = POLICY_F, H = POLICY_H;
  fill(0, F, H, 0x5031);
  fill(F * H + H, H, H, 0x5032);
  fill(F * H + H + H * H + H, H, 1, 0x5033);
  CK(cudaMemcpyAsync(params_, p.data(), POLICY_PARAMS * 4, cudaMemcpyHostToDevice, st_));
  CK(cudaEventCreate(&pev_[0]));
  CK(cudaEventCreate(&pev_[1]));
  sync_check("policy alloc");
  policy_bytes_ = np * (POLICY_F * 2 + 16 + 1 + 12) + 4ull * POLICY_PARAMS * 4;
}

void Engine::set_cache_policy(uint32_t policy) {
  check_loaded();
  if (policy != DYCG_CACHE_HOTNESS && policy != DYCG_CACHE_LEARNED)
    throw Error(DYCG_EINVAL, "switchable policies: DYCG_CACHE_HOTNESS, DYCG_CACHE_LEARNED");
  if (!cache_slots_) throw Error(DYCG_ESTATE, "no HBM page cache (budget or policy NONE at create)");
  if (policy == DYCG_CACHE_LEARNED) policy_alloc();
  policy_ = policy;
  drop_graphs();
}

void Engine::policy_trace(uint32_t snapshots) {
  check_loaded();
  policy_alloc();
  if (tx_) cudaFree(tx_);
  if (ty_) cudaFree(ty_);
  tx_ = nullptr;
  ty_ = nullptr;
  trace_cap_ = trace_n_ = trace_post_ = 0;
  if (!snapshots) return;
  CK(cudaMalloc(&tx_, (u64)snapshots * npages_ * POLICY_F * 2));
  CK(cudaMalloc((void **)&ty_, (u64)snapshots * npages_ * 4));
  trace_cap_ = snapshots;
  drop_graphs();
}

// Features of the snapshot being applied (after its mutation, before its
// repair); under the learned policy, admit the pages the network ranks
// highest. Everything runs on the device (no host synchronisation), so the
// same sequence is recorded into the replayed snapshot graphs (capture: no
// stage events, no trace recording).
void Engine::policy_prefetch(size_t nd, size_t na, bool capture) {
  const u64 np = npages_;
  if (!capture) CK(cudaEventRecord(pev_[0], st_));
  CK(cudaMemsetAsync(pdelta_, 0, np * 4, st_));
  // the row-layout features (rows per page, longest row) drift slowly with
  // relocations: refreshed every 8th snapshot (counter on the device)
  CK(launch_page_rows_clear(prows_, pmax_, npages_, pperiod_, st_));
  CK(launch_page_rows(out_.off, out_.len, n_, out_.page_base, page_shift_, prows_, pmax_, pperiod_,
                      st_));
  if (has_in_)
    CK(launch_page_rows(in_.off, in_.len, n_, in_.page_base, page_shift_, prows_, pmax_, pperiod_,
                        st_));
  CK(launch_period_step(pperiod_, st_));
  if (nd) {
    CK(launch_page_delta(k_del_out_, (uint32_t)nd, out_.off, out_.page_base, page_shift_, pdelta_,
                         st_));
    if (has_in_)
      CK(launch_page_delta(k_del_in_, (uint32_t)nd, in_.off, in_.page_base, page_shift_, pdelta_,
                           st_));
  }
  if (na) {
    CK(launch_page_delta(k_add_out_, (uint32_t)na, out_.off, out_.page_base, page_shift_, pdelta_,
                         st_));
    if (has_in_)
      CK(launch_page_delta(k_add_in_, (uint32_t)na, in_.off, in_.page_base, page_shift_, pdelta_,
                           st_));
  }
  CK(launch_features(page_hits_, hist_, age_, pdelta_, prows_, pmax_, npages_, feat_, st_));
  launches_ += 5 + (has_in_ ? 1 : 0) + (nd ? 1 : 0) * (has_in_ ? 2 : 1) +
               (na ? 1 : 0) * (has_in_ ? 2 : 1);
  trace_pending_ = !capture && trace_n_ < trace_cap_;
  if (trace_pending_) {
    CK(cudaMemcpyAsync((char *)tx_ + (u64)trace_n_ * np * POLICY_F * 2, feat_,
                       np * POLICY_F * 2, cudaMemcpyDeviceToDevice, st_));
    CK(cudaMemsetAsync(ty_ + (u64)trace_n_ * np, 0, np * 4, st_));
  }
  if (policy_ == DYCG_CACHE_LEARNED && cache_slots_) {
    CK(launch_mlp_infer(feat_, npages_, params_, cwk_.score, cwk_.ids, &ctl_->err, st_));
    // admit a page only when its predicted reads over the training horizon
    // (log1p of slot reads) pay back at least half of its fill: a fill moves
    // all 2^page_shift slots over the host link, a cached read saves one slot;
    // at most cache_slots / learned_cap_div_ per snapshot (no refresh gate)
    const float payback = std::log1p((float)(1u << page_shift_) * 0.5f);
    CK(cache_rank_given(cwk_, npages_, cache_slots_, payback, page_slot_, st_));
    CachePages pg{out_.d_dst, has_in_ ? in_.d_dst : nullptr, out_.pages, page_shift_,
                  out_.stride, cdst_};
    const uint32_t cap = std::max<uint32_t>(cache_slots_ / learned_cap_div_, 256u);
    CK(cache_apply(cwk_, npages_, 1, cap, page_slot_, free_list_, pg,
                   &ctl_->stat[ST_PAGES_LOADED], &ctl_->stat[ST_PAGES_EVICTED], st_));
    launches_ += 9;
  }
  if (!capture) {
    CK(cudaEventRecord(pev_[1], st_));
    prefetched_ = true;
  }
}

void Engine::policy_train(uint32_t epochs, float lr, uint32_t batch, uint64_t seed,
                          dycg_policy_report *rep) {
  check_loaded();
  if (!trace_n_) throw Error(DYCG_ESTATE, "no access traces recorded (dycg_policy_trace)");
  if (batch == 0 || !(lr > 0.f)) throw Error(DYCG_EINVAL, "batch and lr must be positive");
  // traced snapshots whose target horizon is complete (at least one)
  const int64_t complete = (int64_t)trace_n_ + trace_post_ - POLICY_HORIZON + 1;
  const uint32_t usable = (uint32_t)std::max<int64_t>(1, std::min<int64_t>(trace_n_, complete));
  const u64 total = (u64)usable * npages_;
  float *ylog = nullptr;
  CK(cudaMalloc((void **)&ylog, total * 4));
  struct Free {
    float *p;
    ~Free() { cudaFree(p); }
  } fy{ylog};
  CK(launch_log1p(ty_, ylog, total, st_));
  auto eval = [&]() {
    CK(cudaMemsetAsync(ploss_, 0, 4, st_));
    for (u64 o = 0; o < total; o += (1ull << 30)) {
      const uint32_t c = (uint32_t)std::min<u64>(1ull << 30, total - o);
      CK(launch_mlp_grad((const char *)tx_ + o * POLICY_F * 2, ylog + o, c, c, 0, params_, 0.f,
                         grad_, ploss_, &ctl_->err, st_));
    }
    CK(cudaMemsetAsync(grad_, 0, POLICY_PARAMS * 4, st_));
    float l = 0;
    CK(cudaMemcpyAsync(&l, ploss_, 4, cudaMemcpyDeviceToHost, st_));
    sync_check("policy eval");
    return l / (float)total;
  };
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, st_));
  const float l0 = eval();
  const u64 steps = std::max<u64>(1, (u64)epochs * total / batch);
  for (u64 s = 0; s < steps; s++) {
    CK(launch_mlp_grad(tx_, ylog, total, batch, mix64(seed + s + 1) | 1, params_, 2.f / batch,
                       grad_, ploss_, &ctl_->err, st_));
    CK(launch_adam(params_, grad_, adam_m_, adam_v_, lr, ++adam_step_, st_));
  }
  const float l1 = eval();
  CK(cudaEventRecord(b, st_));
  sync_check("policy train");
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->samples = total;
    rep->steps = steps;
    rep->loss_before = l0;
    rep->loss_after = l1;
    rep->ms = ms;
  }
}

void Engine::policy_params(float *out) {
  policy_alloc();
  CK(cudaMemcpyAsync(out, params_, POLICY_PARAMS * 4, cudaMemcpyDeviceToHost, st_));
  sync_check("policy params");
}

void Engine::policy_set_params(const float *in) {
  policy_alloc();
  CK(cudaMemcpyAsync(params_, in, POLICY_PARAMS * 4, cudaMemcpyHostToDevice, st_));
  sync_check("policy set params");
}

void Engine::sample_row_edges(const uint32_t *sources, uint64_t count, uint64_t seed,
                              dycg_edge *out) {
  check_loaded();
  if (!count) return;
  uint32_t *d_src = nullptr, *d_out = nullptr;
  CK(cudaMalloc(&d_src, count * 4));
  const cudaError_t e0 = cudaMalloc(&d_out, count * 12);
  if (e0 != cudaSuccess) {
    cudaFree(d_src);
    CK(e0);
  }
  cudaError_t e = cudaMemcpyAsync(d_src, sources, count * 4, cudaMemcpyHostToDevice, st_);
  if (e == cudaSuccess) e = dycg::sample_row_edges(adj(out_), d_src, count, seed, n_, d_out, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, count * 12, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  cudaFree(d_src);
  cudaFree(d_out);
  CK(e);
}

void Engine::cache_maintenance(bool initial, dycg_batch_stats *stats) {
  check_loaded();
  if (feat_ && !initial) {
    // page-read history for the learned policy; this snapshot's reads go into
    // the raw targets of the traced snapshots whose horizon covers it: the
    // current snapshot is number c in trace order (traced or not)
    TargetRefs tg{};
    const int64_t traced = (int64_t)trace_n_ + (trace_pending_ ? 1 : 0);
    const int64_t c = trace_pending_ ? (int64_t)trace_n_ : (int64_t)trace_n_ + trace_post_;
    for (int j = 0; j < POLICY_HORIZON; j++) {
      const int64_t k = c - j;
      if (k >= 0 && k < traced) tg.t[j] = ty_ + (u64)k * npages_;
    }
    const bool clear = policy_ != DYCG_CACHE_HOTNESS || !cache_slots_;
    CK(launch_history(page_hits_, hist_, age_, npages_, tg, clear, st_));
    launches_++;
    if (trace_pending_) {
      trace_n_++;
      trace_post_ = 0;
    } else if (trace_post_ < POLICY_HORIZON) {
      trace_post_++;
    }
    trace_pending_ = false;
  }
  if (policy_ == DYCG_CACHE_LEARNED && !initial) {
    // admission ran before the repair (policy_prefetch); the call ends here
    CK(cudaEventRecord(ev_[5], st_));
    if (prefetched_ && stats) {
      CK(cudaMemcpyAsync(cwk_.h_plan, cwk_.plan, sizeof(CachePlan), cudaMemcpyDeviceToHost, st_));
      sync_check("learned maintenance");
      float ms = 0;
      cudaEventElapsedTime(&ms, pev_[0], pev_[1]);
      stats->ms_cache = ms;
      const CachePlan &pl = *cwk_.h_plan;
      stats->cache_pages_loaded = pl.admit;
      stats->cache_pages_evicted = pl.evict;
      const u64 page_bytes = (4ull << page_shift_) * out_.stride;
      stats->link_bytes += (u64)pl.admit * page_bytes;
      stats->hbm_adj_bytes += (u64)pl.admit * page_bytes;
    }
    prefetched_ = false;
    return;
  }
  prefetched_ = false;
  if (!cache_slots_) {
    CK(cudaMemsetAsync(page_hits_, 0, (u64)npages_ * 4, st_));
    return;
  }
  CK(cudaEventRecord(ev_[4], st_));
  // the staging (eviction, fills) of a later round runs on the side stream,
  // hidden behind the next snapshot's record staging and ingest
  hotness_round(initial, !initial);
  CK(cudaEventRecord(ev_[5], st_));
  CK(cudaMemcpyAsync(cwk_.h_plan, cwk_.plan, sizeof(CachePlan), cudaMemcpyDeviceToHost, st_));
  sync_check("cache apply");
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev_[4], ev_[5]);
    const CachePlan &pl = *cwk_.h_plan;
    stats->ms_cache = ms;
    stats->cache_pages_loaded = pl.admit;
    stats->cache_pages_evicted = pl.evict;
    const u64 page_bytes = (4ull << page_shift_) * out_.stride;
    stats->link_bytes += (u64)pl.admit * page_bytes;
    stats->hbm_adj_bytes += (u64)pl.admit * page_bytes;
  }
}

// One hotness round on the device: decayed page scores, top-K ranking, the
// refresh gate, eviction and staging. A page must have been read at least
// kMinScore times (decayed) before it displaces a resident one, so single
// random probes do not churn the cache; the initial load admits the whole
// top K.
void Engine::hotness_round(bool initial, bool side) {
  const float kMinScore = initial ? 0.f : 64.f;
  CK(cache_rank(cwk_, npages_, cache_slots_, 0.75f, kMinScore, page_slot_, st_));
  const uint32_t gate = initial ? 1u : std::max<uint32_t>(1u, cache_slots_ / 1024);
  const uint32_t cap = initial ? cache_slots_ : std::max<uint32_t>(cache_slots_ / 512, 64u);
  CachePages pg{out_.d_dst, has_in_ ? in_.d_dst : nullptr, out_.pages, page_shift_, out_.stride,
                cdst_};
  CK(cache_plan(cwk_, npages_, gate, cap, &ctl_->stat[ST_PAGES_LOADED],
                &ctl_->stat[ST_PAGES_EVICTED], st_));
  if (side) {
    // staging on the side stream, after the plan; the engine stream goes on
    CK(cudaEventRecord(fev_[0], st_));
    CK(cudaStreamWaitEvent(fst_, fev_[0], 0));
    CK(cache_stage(cwk_, npages_, page_slot_, free_list_, pg, fst_));
    CK(cudaEventRecord(fev_[1], fst_));
    staging_ = true;
  } else {
    CK(cache_stage(cwk_, npages_, page_slot_, free_list_, pg, st_));
  }
  launches_ += 9;
}

// Per-snapshot cache maintenance recorded into a replayed snapshot graph:
// the learned policy's page history (its admission ran before the repair),
// or a hotness round, or for an engine without cache the counter reset.
void Engine::maintenance_device() {
  if (feat_) {
    const bool clear = policy_ != DYCG_CACHE_HOTNESS || !cache_slots_;
    CK(launch_history(page_hits_, hist_, age_, npages_, TargetRefs{}, clear, st_));
    launches_++;
  }
  if (policy_ == DYCG_CACHE_LEARNED) return;
  if (!cache_slots_) {
    CK(cudaMemsetAsync(page_hits_, 0, (u64)npages_ * 4, st_));
    return;
  }
  hotness_round(false);
}

void Engine::gather(uint32_t *values, uint32_t *parents) {
  check_loaded();
  if (opt_.algo == DYCG_ALGO_PR) throw Error(DYCG_EINVAL, "PR results: use dycg_gather_ranks");
  if (nq_) {
    gather_query(0, values, parents);
    return;
  }
  std::vector<u64> k(n_);
  CK(cudaMemcpyAsync(k.data(), key_, (u64)n_ * 8, cudaMemcpyDeviceToHost, st_));
  sync_check("gather");
  for (uint32_t v = 0; v < n_; v++) {
    const uint32_t val = key_value(k[v]);
    const uint32_t p1 = key_parent1(k[v]);
    if (values) values[v] = val;
    if (parents) parents[v] = (val == INF32 || p1 == 0) ? INF32 : p1 - 1;
  }
}

void Engine::gather_ranks(float *ranks, float *residuals) {
  check_loaded();
  if (opt_.algo != DYCG_ALGO_PR) throw Error(DYCG_EINVAL, "not a PageRank engine");
  if (ranks) CK(cudaMemcpyAsync(ranks, x_, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  if (residuals) CK(cudaMemcpyAsync(residuals, r_, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  sync_check("gather ranks");
}

// Host bitmap words covering slots [first, first + count) of arena A.
static std::vector<uint32_t> fetch_bits(const Arena &A, u64 first, u64 count, cudaStream_t st) {
  const u64 w0 = first >> 5, w1 = (first + count + 31) >> 5;
  std::vector<uint32_t> b(w1 - w0 + 1, 0);
  if (w1 > w0) cudaMemcpyAsync(b.data(), A.tbits + w0, (w1 - w0) * 4, cudaMemcpyDeviceToHost, st);
  return b;
}

void Engine::get_row(uint32_t v, int incoming, uint32_t *dst, uint32_t *w, uint32_t cap,
                     uint32_t *deg) {
  check_loaded();
  if (v >= n_) throw Error(DYCG_EINVAL, "vertex out of range");
  const Arena &A = (incoming && has_in_) ? in_ : out_;
  u64 off = 0;
  uint32_t len = 0;
  CK(cudaMemcpyAsync(&off, A.off + v, 8, cudaMemcpyDeviceToHost, st_));
  CK(cudaMemcpyAsync(&len, A.len + v, 4, cudaMemcpyDeviceToHost, st_));
  sync_check("row");
  std::vector<uint32_t> bits = fetch_bits(A, off, len, st_);
  sync_check("row bits");
  const u64 w0 = off >> 5;
  uint32_t k = 0;
  for (uint32_t s = 0; s < len; s++) {
    const u64 p = off + s;
    const uint32_t d = A.h_dst[p * A.stride];
    if ((d & TOMB) || ((bits[(p >> 5) - w0] >> (p & 31)) & 1u)) continue;
    if (k < cap) {
      if (dst) dst[k] = d;
      if (w) w[k] = A.stride == 2 ? A.h_dst[p * 2 + 1] : 0u;
    }
    k++;
  }
  if (deg) *deg = k;
}

void Engine::export_csr(uint64_t *off, uint32_t *dst, uint32_t *w) {
  check_loaded();
  std::vector<u64> o(n_);
  std::vector<uint32_t> l(n_);
  CK(cudaMemcpyAsync(o.data(), out_.off, (u64)n_ * 8, cudaMemcpyDeviceToHost, st_));
  CK(cudaMemcpyAsync(l.data(), out_.len, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  std::vector<uint32_t> bits = fetch_bits(out_, 0, out_.slots, st_);
  sync_check("export");
  u64 q = 0;
  for (uint32_t v = 0; v < n_; v++) {
    off[v] = q;
    for (uint32_t s = 0; s < l[v]; s++) {
      const u64 p = o[v] + s;
      const uint32_t d = out_.h_dst[p * out_.stride];
      if ((d & TOMB) || ((bits[p >> 5] >> (p & 31)) & 1u)) continue;
      if (dst) dst[q] = d;
      if (w) w[q] = out_.stride == 2 ? out_.h_dst[p * 2 + 1] : 0u;
      q++;
    }
  }
  off[n_] = q;
}

void Engine::info(dycg_graph_info *out) {
  check_loaded();
  std::memset(out, 0, sizeof(*out));
  out->nodes = n_;
  std::vector<uint32_t> l(n_);
  CK(cudaMemcpyAsync(l.data(), out_.live, (u64)n_ * 4, cudaMemcpyDeviceToHost, st_));
  u64 top_out = 0, top_in = 0;
  CK(cudaMemcpyAsync(&top_out, out_.top, 8, cudaMemcpyDeviceToHost, st_));
  if (has_in_) CK(cudaMemcpyAsync(&top_in, in_.top, 8, cudaMemcpyDeviceToHost, st_));
  if (cache_slots_)
    CK(cudaMemcpyAsync(cwk_.h_plan, cwk_.plan, sizeof(CachePlan), cudaMemcpyDeviceToHost, st_));
  sync_check("info");
  u64 m = 0;
  for (uint32_t x : l) m += x;
  out->live_edges = m;
  out->arena_slots = out_.slots + (has_in_ ? in_.slots : 0);
  out->arena_used = top_out + top_in;
  out->pages = npages_;
  out->cache_slots = cache_slots_;
  out->cached_pages = cache_slots_ ? cache_slots_ - cwk_.h_plan->free_count : 0;
  out->host_bytes = out->arena_slots * 4 * out_.stride;
  out->device_bytes = (u64)n_ * (8 + 4 * 6) + (u64)n_ * (has_in_ ? 48 : 24) +
                      ((u64)cache_slots_ << page_shift_) * 4 * out_.stride + index_bytes_ +
                      qbytes_ + policy_bytes_;
  out->reserved[0] = index_bytes_;  // fence index + deletion bitmap (part of the budget)
  out->page_shift = page_shift_;
  out->has_incoming = has_in_ ? 1 : 0;
}

void Engine::sample_edges(uint64_t count, uint64_t seed, dycg_edge *out) {
  check_loaded();
  if (!count) return;
  const uint32_t n = n_;
  u64 *pre = nullptr;
  CK(cudaMalloc(&pre, (n + 1ull) * 8));
  size_t tb = 0;
  CK(build_scan_u32_to_u64(nullptr, tb, out_.live, pre, n, st_));
  void *temp = nullptr;
  CK(cudaMalloc(&temp, std::max<size_t>(tb, 16)));
  CK(build_scan_u32_to_u64(temp, tb, out_.live, pre, n, st_));
  u64 last_pre = 0;
  uint32_t last_live = 0;
  CK(cudaMemcpyAsync(&last_pre, pre + n - 1, 8, cudaMemcpyDeviceToHost, st_));
  CK(cudaMemcpyAsync(&last_live, out_.live + n - 1, 4, cudaMemcpyDeviceToHost, st_));
  sync_check("sample scan");
  cudaFree(temp);
  const u64 total = last_pre + last_live;
  if (count > total) {
    cudaFree(pre);
    throw Error(DYCG_EINVAL, "more samples requested than live edges");
  }
  // draw with oversampling, keep the first `count` distinct ranks in draw order
  std::vector<u64> chosen;
  chosen.reserve(count);
  std::unordered_set<u64> seen;
  seen.reserve(count * 2);
  u64 round = 0;
  while (chosen.size() < count) {
    const u64 draws = (count - chosen.size()) + (count - chosen.size()) / 16 + 64;
    u64 *pos = nullptr;
    CK(cudaMalloc(&pos, draws * 8));
    CK(sample_draw(pos, draws, mix64(seed + round * 0x9E37ull), total, st_));
    std::vector<u64> h(draws);
    CK(cudaMemcpyAsync(h.data(), pos, draws * 8, cudaMemcpyDeviceToHost, st_));
    sync_check("sample draw");
    cudaFree(pos);
    for (u64 r : h) {
      if (chosen.size() >= count) break;
      if (seen.insert(r).second) chosen.push_back(r);
    }
    if (++round > 64) break;
  }
  const u64 k = chosen.size();
  u64 *pos = nullptr;
  uint32_t *res = nullptr;
  CK(cudaMalloc(&pos, k * 8));
  CK(cudaMalloc(&res, k * 12));
  CK(cudaMemcpyAsync(pos, chosen.data(), k * 8, cudaMemcpyHostToDevice, st_));
  CK(sample_resolve(pos, k, pre, n, adj(out_), res, st_));
  CK(cudaMemcpyAsync(out, res, k * 12, cudaMemcpyDeviceToHost, st_));
  sync_check("sample resolve");
  cudaFree(pos);
  cudaFree(res);
  cudaFree(pre);
  if (k < count) throw Error(DYCG_ELIMIT, "could not draw enough distinct edges");
}

}  // namespace dycg
