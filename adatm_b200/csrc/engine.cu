// engine.cu -- tensor + plan + trees + memo rows + factors + CP-ALS sweep.
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace adatm {

namespace {
// Host workers for the factor conversions at the C-ABI boundary, started
// once: starting threads on every call costs more than the conversion. A
// call splits rows [0, rows) into parts, runs part 0 itself and waits for the
// rest; calls are serialised.
class HostPool {
 public:
  static HostPool &instance() {
    static HostPool *p = new HostPool();  // never destroyed: its workers are detached
    return *p;
  }
  void run(uint64_t rows, unsigned parts, const std::function<void(uint64_t, uint64_t)> &f) {
    parts = std::min<unsigned>(parts, nworkers_ + 1);
    if (parts <= 1 || rows < 2) {
      f(0, rows);
      return;
    }
    std::lock_guard<std::mutex> one(call_mu_);
    const uint64_t step = (rows + parts - 1) / parts;
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &f;
      rows_ = rows;
      step_ = step;
      left_ = parts - 1;
      next_ = 1;
      parts_ = parts;
    }
    cv_.notify_all();
    f(0, std::min(rows, step));
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return left_ == 0; });
    parts_ = 0;
    next_ = 0;
    fn_ = nullptr;
  }

 private:
  HostPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    nworkers_ = std::min(15u, hw > 1 ? hw - 1 : 0u);
    for (unsigned t = 0; t < nworkers_; ++t) std::thread([this] { loop(); }).detach();
  }
  void loop() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return next_ < parts_; });
      while (next_ < parts_) {
        const unsigned p = next_++;
        const auto *fn = fn_;
        const uint64_t a = p * step_, b = std::min(rows_, a + step_);
        lk.unlock();
        if (a < b) (*fn)(a, b);
        lk.lock();
        if (--left_ == 0) done_.notify_one();
      }
    }
  }
  unsigned nworkers_ = 0;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_;
  const std::function<void(uint64_t, uint64_t)> *fn_ = nullptr;
  uint64_t rows_ = 0, step_ = 0;
  unsigned parts_ = 0, next_ = 0, left_ = 0;
};

// Rows [0, rows) of a host conversion, split over the pool when large.
template <typename F>
void host_rows(uint64_t rows, uint64_t row_elems, F &&f) {
  const unsigned parts = (unsigned)std::min<uint64_t>(16, rows * row_elems / 32768 + 1);
  HostPool::instance().run(rows, parts, std::function<void(uint64_t, uint64_t)>(f));
}

int depth_of(const DevCsf &c, int mode) {
  for (int l = 0; l < c.nmodes; ++l)
    if ((int)c.dim_perm[l] == mode) return l;
  throw BadInput("mode missing from the tree's level order");
}
}  // namespace

Engine::Engine(std::shared_ptr<const DevCoo> coo, std::vector<std::shared_ptr<DevCsf>> trees,
               uint64_t rank, const Plan &plan, const EngineOptions &opt, cudaStream_t stream)
    : coo_(std::move(coo)), R_(rank), ldr_(ldr_of(rank)), plan_(plan), opt_(opt),
      stream_(stream), csf_(std::move(trees)) {
  const int N = coo_->nmodes;
  if (rank == 0 || rank > 128) throw BadInput("rank must be 1..128");
  if (csf_.empty()) {
    for (int g = 0; g < plan_.n_csf; ++g) {
      csf_.emplace_back(std::make_shared<DevCsf>());
      csf_build(*coo_, plan_.tree(g).o_opt, *csf_.back(), stream_);
    }
  }
  if ((int)csf_.size() != plan_.n_csf) throw BadInput("tree count does not match the plan");
  for (int g = 0; g < plan_.n_csf; ++g) {
    const Group &gp = plan_.tree(g);
    for (uint64_t deg = 0; deg < gp.n_imten; ++deg) {
      const uint64_t lvl = gp.begin_imten - 1 - deg;
      const size_t n = (size_t)csf_[g]->nfibs[lvl] * ldr_;
      memo_[g][deg].alloc(n);
      ADATM_CUDA(cudaMemsetAsync(memo_[g][deg].get(), 0, n * sizeof(float), stream_));
    }
  }
  uint64_t maxdim = 1;
  for (int m = 0; m < N; ++m) {
    maxdim = std::max(maxdim, coo_->dims[m]);
    A_[m].alloc((size_t)coo_->dims[m] * ldr_);
    ADATM_CUDA(cudaMemsetAsync(A_[m].get(), 0, A_[m].bytes(), stream_));
    if (opt_.factor_type == FactorType::BF16) {
      Ab_[m].alloc((size_t)coo_->dims[m] * ldr_);
      ADATM_CUDA(cudaMemsetAsync(Ab_[m].get(), 0, Ab_[m].bytes(), stream_));
    }
    G_[m].alloc((size_t)R_ * R_);
  }
  M_.alloc((size_t)maxdim * ldr_);
  int sms = 148;
  {
    int dev = 0;
    ADATM_CUDA(cudaGetDevice(&dev));
    ADATM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  w_.init(N, (int)R_, 2 * sms, opt_.max_iters);
  ADATM_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  ADATM_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  ADATM_CUDA(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
  ADATM_CUDA(cudaEventCreateWithFlags(&staged_, cudaEventDisableTiming));
  ADATM_CUDA(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  for (auto &ev : updated_) ADATM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  for (auto &ev : landed_) ADATM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  build_walks();
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

Engine::~Engine() {
  if (staged_pending_) cudaEventSynchronize(staged_);
  drop_graph();
  if (join_) cudaEventDestroy(join_);
  if (fork_) cudaEventDestroy(fork_);
  if (staged_) cudaEventDestroy(staged_);
  if (copy_) cudaStreamSynchronize(copy_);
  for (auto ev : updated_)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : landed_)
    if (ev) cudaEventDestroy(ev);
  if (copy_) cudaStreamDestroy(copy_);
  if (side_) cudaStreamDestroy(side_);
  if (staging_) cudaFreeHost(staging_);
}

void Engine::drop_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
}

void Engine::set_chunks(uint32_t chunk_leaf, uint32_t chunk_rows) {
  if (chunk_leaf == 0 || chunk_rows == 0) throw BadInput("chunk sizes must be positive");
  drop_graph();
  opt_.chunk_leaf = chunk_leaf;
  opt_.chunk_rows = chunk_rows;
  build_walks();
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::set_deterministic(bool on) {
  if (on == opt_.deterministic) return;
  drop_graph();
  opt_.deterministic = on;
  build_walks();
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::set_walkers(int walkers) {
  if (walkers != 0 && !walkers_supported((int)R_, walkers))
    throw BadInput("no contraction kernel for " + std::to_string(walkers) + " walkers at rank " +
                   std::to_string(R_));
  drop_graph();
  opt_.walkers = walkers;
  for (int m = 0; m < coo_->nmodes; ++m) {
    walk_[m]->walkers = walkers;
    if (direct_[m]) direct_[m]->walkers = walkers;
  }
  for (auto &kv : custom_) kv.second->walkers = walkers;
}

void Engine::set_fold(int fold) {
  if (fold < -1 || fold > 2) throw BadInput("folded levels must be -1 (automatic), 0, 1 or 2");
  drop_graph();
  opt_.fold = fold;
  for (int m = 0; m < coo_->nmodes; ++m) {
    walk_[m]->fold = fold;
    if (direct_[m]) direct_[m]->fold = fold;
  }
  for (auto &kv : custom_) kv.second->fold = fold;
}

void Engine::set_resident_grid(bool on) {
  drop_graph();
  opt_.resident_grid = on;
  for (int m = 0; m < coo_->nmodes; ++m) {
    walk_[m]->resident = on;
    if (direct_[m]) direct_[m]->resident = on;
  }
  for (auto &kv : custom_) kv.second->resident = on;
}

float Engine::time_sweeps(int count) {
  cudaEvent_t a, b;
  ADATM_CUDA(cudaEventCreate(&a));
  ADATM_CUDA(cudaEventCreate(&b));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  ADATM_CUDA(cudaEventRecord(a, stream_));
  for (int i = 0; i < count; ++i) sweep();
  ADATM_CUDA(cudaEventRecord(b, stream_));
  ADATM_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  ADATM_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

int Engine::autotune(const std::vector<std::pair<uint32_t, uint32_t>> &options, int sweeps) {
  if (options.empty()) throw BadInput("no chunk options to tune");
  int best = -1;
  float best_ms = 0;
  for (size_t i = 0; i < options.size(); ++i) {
    set_chunks(options[i].first, options[i].second);
    als_begin();
    capture_graph();
    time_sweeps(1);
    const float ms = time_sweeps(std::max(1, sweeps));
    if (best < 0 || ms < best_ms) {
      best = (int)i;
      best_ms = ms;
    }
  }
  set_chunks(options[best].first, options[best].second);
  return best;
}

BatchSweep::BatchSweep(std::vector<Engine *> engines, cudaStream_t stream)
    : e_(std::move(engines)), s_(stream) {
  if (e_.empty()) throw BadInput("an empty batch");
  for (Engine *e : e_)
    if (!e) throw BadInput("a null engine in the batch");
  // the branches' walks run side by side: one chunk per warp, so their
  // blocks interleave instead of each walk holding every SM in turn
  for (Engine *e : e_) e->set_resident_grid(false);
  ADATM_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  join_.resize(e_.size(), nullptr);
  for (auto &ev : join_) ADATM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
}

BatchSweep::~BatchSweep() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
  for (auto ev : join_)
    if (ev) cudaEventDestroy(ev);
  if (fork_) cudaEventDestroy(fork_);
}

void BatchSweep::begin() {
  for (Engine *e : e_) e->als_begin();
  if (exec_) return;
  ADATM_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
  try {
    ADATM_CUDA(cudaEventRecord(fork_, s_));
    for (size_t i = 0; i < e_.size(); ++i) {
      ADATM_CUDA(cudaStreamWaitEvent(e_[i]->stream(), fork_, 0));
      e_[i]->sweep_eager();
      ADATM_CUDA(cudaEventRecord(join_[i], e_[i]->stream()));
      ADATM_CUDA(cudaStreamWaitEvent(s_, join_[i], 0));
    }
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(s_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  ADATM_CUDA(cudaStreamEndCapture(s_, &graph_));
  ADATM_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

void BatchSweep::sweep() {
  if (!exec_) throw BadInput("the batch has not begun");
  ADATM_CUDA(cudaGraphLaunch(exec_, s_));
}

float BatchSweep::time_sweeps(int count) {
  cudaEvent_t a, b;
  ADATM_CUDA(cudaEventCreate(&a));
  ADATM_CUDA(cudaEventCreate(&b));
  ADATM_CUDA(cudaStreamSynchronize(s_));
  ADATM_CUDA(cudaEventRecord(a, s_));
  for (int i = 0; i < count; ++i) sweep();
  ADATM_CUDA(cudaEventRecord(b, s_));
  ADATM_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  ADATM_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

int BatchSweep::kernels_per_sweep() const {
  int k = 0;
  for (Engine *e : e_) k += e->kernels_per_sweep();
  return k;
}

float *Engine::staging(size_t n) {
  // the host may write the rows only once the copies that read them are done
  if (staged_pending_) {
    ADATM_CUDA(cudaEventSynchronize(staged_));
    staged_pending_ = false;
  }
  if (n > staging_n_) {
    if (staging_) cudaFreeHost(staging_);
    staging_ = nullptr;
    staging_n_ = 0;
    ADATM_CUDA(cudaMallocHost(&staging_, n * sizeof(float)));
    staging_n_ = n;
  }
  return staging_;
}

size_t Engine::memo_bytes() const {
  size_t b = 0;
  for (int g = 0; g < kMaxModes; ++g)
    for (int d = 0; d < kMaxModes; ++d) b += memo_[g][d].bytes();
  return b;
}

size_t Engine::csf_bytes() const {
  size_t b = 0;
  for (auto &c : csf_) b += c->device_bytes();
  return b;
}

// Memo levels a reuse MTTKRP of output level d can start from: the leading
// stored levels of the group that lie below d (mttkrp.c:1578-1588 with
// rcsf_reverse_mode_order, adatm_rcsf.c:313-326).
static uint64_t reuse_indeg(const Group &gp, int d) {
  const uint64_t b = gp.begin_imten;
  uint64_t rd[kMaxModes + 1] = {0};
  uint64_t j = 0;
  for (int64_t i = (int64_t)b; i >= 0; --i)
    if (i != d) rd[j++] = (uint64_t)i;
  uint64_t indeg = 0;
  for (uint64_t i = 0; i < gp.n_imten; ++i)
    if (b - i == rd[i]) ++indeg;
  return indeg;
}

void Engine::check_use(int mode, int tree, int tag) const {
  const int N = coo_->nmodes;
  if (mode < 0 || mode >= N) throw BadInput("mode out of range");
  if (tree < 0 || tree >= (int)csf_.size()) throw BadInput("use_csfs names a tree that was not built");
  const int d = depth_of(*csf_[tree], mode);
  const Group &gp = plan_.tree(tree);
  switch (tag) {
    case 0:
      if (d != 0) throw BadInput("use_tags 0 (root MTTKRP) on a mode that is not the tree's root");
      break;
    case 1:
      if (gp.n_imten == 0) throw BadInput("use_tags 1 (memo reuse) on a tree whose group stores no memo rows");
      // the reference indexes the memo sequence by indeg-1 (mttkrp.c:1591)
      if (reuse_indeg(gp, d) == 0)
        throw BadInput("use_tags 1 (memo reuse) on a mode whose level lies below every stored memo level");
      break;
    case 2:
      if (d == 0) throw BadInput("use_tags 2 (recompute) on the tree's root mode");
      break;
    default: throw BadInput("use_tags must be 0, 1 or 2");
  }
}

std::unique_ptr<TreeWalk> Engine::make_walk(int mode, int g, int tag) {
  const int N = coo_->nmodes;
  const DevCsf &c = *csf_[g];
  const Group &gp = plan_.tree(g);
  const int d = depth_of(c, mode);
  auto w = std::make_unique<TreeWalk>();
  w->csf = &c;
  w->R = (int)R_;
  w->ldr = ldr_;
  w->src = N - 1;
  w->out = d;
  w->chunk = opt_.chunk_leaf;
  w->resident = opt_.resident_grid;
  w->walkers = opt_.walkers;
  w->fold = opt_.fold;
  w->deterministic = opt_.deterministic;
  if (tag == 0 && gp.n_imten > 0) {
    // memo root: store level begin_imten-1-deg into memo tree deg
    for (uint64_t deg = 0; deg < gp.n_imten; ++deg)
      w->store[gp.begin_imten - 1 - deg] = memo_[g][deg].get();
  } else if (tag == 1) {
    const uint64_t indeg = reuse_indeg(gp, d);
    if (indeg > 0) {
      w->src = (int)(gp.begin_imten - indeg);
      w->src_rows = memo_[g][indeg - 1].get();
      w->chunk = opt_.chunk_rows;
    }
  }
  walk_prepare(*w, stream_);
  return w;
}

void Engine::build_walks() {
  custom_.clear();
  for (int m = 0; m < coo_->nmodes; ++m) {
    const int g = (int)plan_.use_csfs[m];
    walk_[m] = make_walk(m, g, (int)plan_.use_tags[m]);
    direct_[m].reset();  // built on first use (mttkrp_direct)
  }
}

void Engine::set_use(const uint64_t *use_csfs, const uint64_t *use_tags) {
  const int N = coo_->nmodes;
  bool same = true;
  for (int m = 0; m < N; ++m) {
    check_use(m, (int)std::min<uint64_t>(use_csfs[m], kMaxModes),
              (int)std::min<uint64_t>(use_tags[m], 3));
    if (use_tags[m] == 1) {
      bool root_before = false;
      for (int k = 0; k < m; ++k) root_before |= use_csfs[k] == use_csfs[m] && use_tags[k] == 0;
      if (!root_before)
        throw BadInput("use_tags 1 (memo reuse) needs the root MTTKRP (tag 0) of the same tree at an "
                       "earlier mode of the sweep");
    }
    same &= plan_.use_csfs[m] == use_csfs[m] && plan_.use_tags[m] == use_tags[m];
  }
  if (same) return;
  drop_graph();
  for (int m = 0; m < N; ++m) {
    plan_.use_csfs[m] = use_csfs[m];
    plan_.use_tags[m] = use_tags[m];
  }
  build_walks();
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::mttkrp_with(int mode, int tree, int tag, double *out) {
  check_use(mode, tree, tag);
  const TreeWalk *w = nullptr;
  if ((int)plan_.use_csfs[mode] == tree && (int)plan_.use_tags[mode] == tag) {
    w = walk_[mode].get();
  } else {
    auto &slot = custom_[std::make_tuple(mode, tree, tag)];
    if (!slot) slot = make_walk(mode, tree, tag);
    w = slot.get();
  }
  ADATM_CUDA(cudaMemsetAsync(out, 0, (size_t)coo_->dims[mode] * ldr_ * sizeof(double), stream_));
  walk_launch(*w, level_factors(tree, opt_.factor_type), opt_.factor_type, out, stream_);
}

LevelFactors Engine::level_factors(int g, FactorType ft) const {
  LevelFactors f;
  const DevCsf &c = *csf_[g];
  for (int l = 0; l < c.nmodes; ++l) {
    const int m = (int)c.dim_perm[l];
    f.U[l] = ft == FactorType::BF16 ? (const void *)Ab_[m].get() : (const void *)A_[m].get();
  }
  return f;
}

void Engine::mttkrp_as(int mode, double *out, FactorType ft) {
  ADATM_CUDA(cudaMemsetAsync(out, 0, (size_t)coo_->dims[mode] * ldr_ * sizeof(double), stream_));
  walk_launch(*walk_[mode], level_factors((int)plan_.use_csfs[mode], ft), ft, out, stream_);
}

void Engine::mttkrp(int mode, double *out) { mttkrp_as(mode, out, opt_.factor_type); }

FactorType Engine::sweep_type(int mode) const {
  // With BF16 factors every factor value is BF16-representable (the update
  // rounds both copies, and the Grams are taken from the rounded rows), so
  // every walk gathers the half-width rows and sees exactly the factor the
  // normal equations and the fit use.
  (void)mode;
  return opt_.factor_type;
}

void Engine::mttkrp_direct(int mode, double *out) {
  ADATM_CUDA(cudaMemsetAsync(out, 0, (size_t)coo_->dims[mode] * ldr_ * sizeof(double), stream_));
  if (!direct_[mode]) direct_[mode] = make_walk(mode, (int)plan_.use_csfs[mode], 2);
  walk_launch(*direct_[mode], level_factors((int)plan_.use_csfs[mode], opt_.factor_type),
              opt_.factor_type, out, stream_);
}

int Engine::kernels_per_mttkrp(int mode) const { return walk_kernels(*walk_[mode]); }

int Engine::kernels_per_sweep() const {
  int k = 1;  // fit
  // per mode: the walks, the Gram inverse, the update, its finalize, the
  // scale; BF16 factors add the Gram of the rounded rows (two kernels)
  const int dense = opt_.factor_type == FactorType::BF16 ? 6 : 4;
  for (int m = 0; m < coo_->nmodes; ++m) k += kernels_per_mttkrp(m) + dense;
  return k;
}

double Engine::mttkrp_bytes(int mode) const {
  const TreeWalk &w = *walk_[mode];
  uint64_t dl[kMaxModes] = {0};
  for (int l = 0; l < w.csf->nmodes; ++l) dl[l] = coo_->dims[w.csf->dim_perm[l]];
  return walk_compulsory_bytes(w, sweep_type(mode), dl, coo_->dims[mode]);
}

void Engine::init_factors(uint64_t seed) {
  for (int m = 0; m < coo_->nmodes; ++m)
    factor_init_device(A_[m].get(), Ab_[m].get(), coo_->dims[m], (int)R_, ldr_, seed, (uint64_t)m,
                       stream_);
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::set_factors(const double *const *host) {
  const int N = coo_->nmodes;
  size_t total = 0, offs[kMaxModes];
  for (int m = 0; m < N; ++m) {
    offs[m] = total;
    total += (size_t)coo_->dims[m] * ldr_;
  }
  float *buf = staging(total);
  // largest mode first: each mode's copy runs while the next is converted,
  // so the sweep waits only on the last (smallest) one
  int order[kMaxModes];
  for (int m = 0; m < N; ++m) order[m] = m;
  std::stable_sort(order, order + N, [&](int x, int y) { return coo_->dims[x] > coo_->dims[y]; });
  for (int k = 0; k < N; ++k) {
    const int m = order[k];
    const uint64_t I = coo_->dims[m];
    float *b = buf + offs[m];
    const double *h = host[m];
    const uint64_t R = R_, L = (uint64_t)ldr_;
    host_rows(I, L, [=](uint64_t i0, uint64_t i1) {
      for (uint64_t i = i0; i < i1; ++i) {
        for (uint64_t r = 0; r < R; ++r) b[i * L + r] = (float)h[i * R + r];
        for (uint64_t r = R; r < L; ++r) b[i * L + r] = 0.f;
      }
    });
    ADATM_CUDA(cudaMemcpyAsync(A_[m].get(), b, (size_t)I * ldr_ * sizeof(float),
                               cudaMemcpyHostToDevice, stream_));
    if (Ab_[m].get()) to_bf16(A_[m].get(), Ab_[m].get(), I, ldr_, stream_);
  }
  // the copies run on; the staging rows are not reused before they end
  ADATM_CUDA(cudaEventRecord(staged_, stream_));
  staged_pending_ = true;
}

void Engine::get_factors(double *const *host) {
  size_t total = 0;
  for (int m = 0; m < coo_->nmodes; ++m) total += (size_t)coo_->dims[m] * ldr_;
  float *buf = staging(total);
  size_t off = 0;
  for (int m = 0; m < coo_->nmodes; ++m) {
    ADATM_CUDA(cudaMemcpyAsync(buf + off, A_[m].get(), (size_t)coo_->dims[m] * ldr_ * sizeof(float),
                               cudaMemcpyDeviceToHost, stream_));
    off += (size_t)coo_->dims[m] * ldr_;
  }
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  off = 0;
  for (int m = 0; m < coo_->nmodes; ++m) {
    const uint64_t I = coo_->dims[m];
    for (uint64_t i = 0; i < I; ++i)
      for (uint64_t r = 0; r < R_; ++r) host[m][i * R_ + r] = (double)buf[off + i * ldr_ + r];
    off += (size_t)I * ldr_;
  }
}

void Engine::get_normalized(double *const *host, double *lambda) {
  const int N = coo_->nmodes;
  size_t total = 0;
  for (int m = 0; m < N; ++m) total += (size_t)coo_->dims[m] * ldr_;
  // factor rows, then the Grams and lambda (FP64, 8-byte aligned: total is
  // a multiple of 4 floats), all into the pinned staging rows, one sync
  const size_t extra = 2 * ((size_t)N * R_ * R_ + R_);
  float *buf = staging(total + extra);
  double *diag = reinterpret_cast<double *>(buf + total);
  double *lam = diag + (size_t)N * R_ * R_;
  size_t off = 0;
  for (int m = 0; m < N; ++m) {
    ADATM_CUDA(cudaMemcpyAsync(buf + off, A_[m].get(), (size_t)coo_->dims[m] * ldr_ * sizeof(float),
                               cudaMemcpyDeviceToHost, stream_));
    ADATM_CUDA(cudaMemcpyAsync(diag + (size_t)m * R_ * R_, G_[m].get(), R_ * R_ * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_));
    off += (size_t)coo_->dims[m] * ldr_;
  }
  ADATM_CUDA(cudaMemcpyAsync(lam, w_.lambda.get(), R_ * sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  std::memcpy(lambda, lam, R_ * sizeof(double));
  std::vector<double> inv(R_);
  off = 0;
  for (int m = 0; m < N; ++m) {
    const double *G = diag + (size_t)m * R_ * R_;
    for (uint64_t r = 0; r < R_; ++r) {
      const double nrm = std::sqrt(std::max(G[r * R_ + r], 0.0));
      inv[r] = nrm > 0 ? 1.0 / nrm : 0.0;
      lambda[r] *= nrm;
    }
    const uint64_t I = coo_->dims[m];
    const float *b = buf + off;
    double *h = host[m];
    const double *iv = inv.data();
    const uint64_t R = R_, L = (uint64_t)ldr_;
    host_rows(I, R, [=](uint64_t i0, uint64_t i1) {
      for (uint64_t i = i0; i < i1; ++i)
        for (uint64_t r = 0; r < R; ++r) h[i * R + r] = (double)b[i * L + r] * iv[r];
    });
    off += (size_t)I * ldr_;
  }
}

double Engine::sweep_download(double *const *host, double *lambda) {
  const int N = coo_->nmodes;
  sweep();
  size_t total = 0;
  for (int m = 0; m < N; ++m) total += (size_t)coo_->dims[m] * ldr_;
  // the same staging layout as get_normalized: rows, then Grams and lambda
  const size_t extra = 2 * ((size_t)N * R_ * R_ + R_);
  float *buf = staging(total + extra);
  double *diag = reinterpret_cast<double *>(buf + total);
  double *lam = diag + (size_t)N * R_ * R_;
  size_t off = 0;
  for (int m = 0; m < N; ++m) {
    ADATM_CUDA(cudaStreamWaitEvent(copy_, updated_[m], 0));
    ADATM_CUDA(cudaMemcpyAsync(buf + off, A_[m].get(), (size_t)coo_->dims[m] * ldr_ * sizeof(float),
                               cudaMemcpyDeviceToHost, copy_));
    ADATM_CUDA(cudaMemcpyAsync(diag + (size_t)m * R_ * R_, G_[m].get(), R_ * R_ * sizeof(double),
                               cudaMemcpyDeviceToHost, copy_));
    ADATM_CUDA(cudaEventRecord(landed_[m], copy_));
    off += (size_t)coo_->dims[m] * ldr_;
  }
  // lambda is final after the last mode's update, which the copy stream
  // has waited for
  ADATM_CUDA(cudaMemcpyAsync(lam, w_.lambda.get(), R_ * sizeof(double), cudaMemcpyDeviceToHost, copy_));
  ADATM_CUDA(cudaEventRecord(landed_[N], copy_));
  // each mode is normalised as it lands, while the GPU runs the later modes
  std::vector<double> nrm((size_t)N * R_);
  off = 0;
  for (int m = 0; m < N; ++m) {
    ADATM_CUDA(cudaEventSynchronize(landed_[m]));
    const double *G = diag + (size_t)m * R_ * R_;
    std::vector<double> inv(R_);
    for (uint64_t r = 0; r < R_; ++r) {
      const double n = std::sqrt(std::max(G[r * R_ + r], 0.0));
      nrm[(size_t)m * R_ + r] = n;
      inv[r] = n > 0 ? 1.0 / n : 0.0;
    }
    const uint64_t I = coo_->dims[m];
    const float *b = buf + off;
    double *h = host[m];
    const double *iv = inv.data();
    const uint64_t R = R_, L = (uint64_t)ldr_;
    host_rows(I, R, [=](uint64_t i0, uint64_t i1) {
      for (uint64_t i = i0; i < i1; ++i)
        for (uint64_t r = 0; r < R; ++r) h[i * R + r] = (double)b[i * L + r] * iv[r];
    });
    off += (size_t)I * ldr_;
  }
  ADATM_CUDA(cudaEventSynchronize(landed_[N]));
  std::memcpy(lambda, lam, R_ * sizeof(double));
  for (int m = 0; m < N; ++m)
    for (uint64_t r = 0; r < R_; ++r) lambda[r] *= nrm[(size_t)m * R_ + r];
  return fit_host();
}

void Engine::get_lambda(double *host) const {
  ADATM_CUDA(cudaMemcpyAsync(host, w_.lambda.get(), R_ * sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::als_begin() {
  for (int m = 0; m < coo_->nmodes; ++m)
    gram(A_[m].get(), coo_->dims[m], (int)R_, ldr_, G_[m].get(), w_, stream_,
         opt_.factor_type == FactorType::BF16);
  if (!ttnorm_ready_) {
    frob_sq(csf_[0]->vals64.get(), coo_->nnz, w_, stream_);
    ttnorm_ready_ = true;
  }
  ADATM_CUDA(cudaMemsetAsync(w_.iter.get(), 0, sizeof(int), stream_));
  ADATM_CUDA(cudaMemsetAsync(w_.fit_trace.get(), 0, w_.max_trace * sizeof(double), stream_));
}

void Engine::sweep_eager() {
  const int N = coo_->nmodes;
  GramSet gs;
  for (int m = 0; m < kMaxModes; ++m) gs.G[m] = m < N ? G_[m].get() : nullptr;
  for (int m = 0; m < N; ++m) {
    // the Gram inverse of mode m needs only the other modes' Grams, final
    // since mode m-1's update: it runs beside mode m's MTTKRP
    ADATM_CUDA(cudaEventRecord(fork_, stream_));
    ADATM_CUDA(cudaStreamWaitEvent(side_, fork_, 0));
    gram_inverse(gs, m, w_, side_);
    ADATM_CUDA(cudaEventRecord(join_, side_));
    mttkrp_as(m, M_.get(), sweep_type(m));
    ADATM_CUDA(cudaStreamWaitEvent(stream_, join_, 0));
    update_factor(M_.get(), coo_->dims[m], A_[m].get(), Ab_[m].get(), G_[m].get(), m == N - 1, w_,
                  stream_);
    // mode m's rows and Gram are final for this sweep, so a download may
    // start here: an event node when the sweep is being captured (the
    // external flag is refused outside a capture)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ADATM_CUDA(cudaStreamIsCapturing(stream_, &cap));
    if (cap == cudaStreamCaptureStatusActive)
      ADATM_CUDA(cudaEventRecordWithFlags(updated_[m], stream_, cudaEventRecordExternal));
    else
      ADATM_CUDA(cudaEventRecord(updated_[m], stream_));
  }
  fit(gs, w_, stream_);
}

void Engine::mttkrp_into(int mode, double *dev_out) {
  mttkrp_as(mode, dev_out, sweep_type(mode));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::update_from(int mode, const double *dev_M) {
  const int N = coo_->nmodes;
  if (mode < 0 || mode >= N) throw BadInput("mode out of range");
  GramSet gs;
  for (int m = 0; m < kMaxModes; ++m) gs.G[m] = m < N ? G_[m].get() : nullptr;
  gram_inverse(gs, mode, w_, stream_);
  update_factor(dev_M, coo_->dims[mode], A_[mode].get(), Ab_[mode].get(), G_[mode].get(),
                mode == N - 1, w_, stream_);
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

double Engine::fit_step() {
  const int N = coo_->nmodes;
  GramSet gs;
  for (int m = 0; m < kMaxModes; ++m) gs.G[m] = m < N ? G_[m].get() : nullptr;
  fit(gs, w_, stream_);
  return fit_host();
}

double Engine::ttnorm_local() {
  if (!ttnorm_ready_) {
    frob_sq(csf_[0]->vals64.get(), coo_->nnz, w_, stream_);
    ttnorm_ready_ = true;
  }
  double v = 0;
  ADATM_CUDA(cudaMemcpyAsync(&v, w_.scalars.get(), sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  return v;
}

void Engine::set_ttnorm(double v) {
  ttnorm_local();  // keeps als_begin from recomputing it
  ADATM_CUDA(cudaMemcpyAsync(w_.scalars.get(), &v, sizeof(double), cudaMemcpyHostToDevice, stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::capture_graph() {
  if (graph_exec_) return;
  // kernels set their shared-memory attributes on first use: run the
  // attribute paths once outside the capture on scratch state
  ADATM_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  try {
    sweep_eager();
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(stream_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  ADATM_CUDA(cudaStreamEndCapture(stream_, &graph_));
  ADATM_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
}

void Engine::sweep() {
  if (graph_exec_)
    ADATM_CUDA(cudaGraphLaunch(graph_exec_, stream_));
  else
    sweep_eager();
}

double Engine::fit_host() {
  double f = 0;
  ADATM_CUDA(cudaMemcpyAsync(&f, w_.scalars.get() + 1, sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  return f;
}

int Engine::iter_host() {
  int it = 0;
  ADATM_CUDA(cudaMemcpyAsync(&it, w_.iter.get(), sizeof(int), cudaMemcpyDeviceToHost, stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
  return it;
}

void Engine::fit_trace(double *host, int n) {
  n = std::min(n, w_.max_trace);
  ADATM_CUDA(cudaMemcpyAsync(host, w_.fit_trace.get(), n * sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
  ADATM_CUDA(cudaStreamSynchronize(stream_));
}

}  // namespace adatm
