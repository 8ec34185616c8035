// api.cu -- the C ABI: SPLATT's public functions, AdaTM's entry points and
// the device-resident B200 interface (include/splatt.h, include/adatm_b200.h).
//
// Host-visible trees (splatt_csf) keep the reference layout and live in host
// memory like the reference's; their device mirrors (COO, trees, engines per
// rank) are kept in a registry keyed by the address of the splatt_csf array
// the library returned, and released by splatt_free_csf.
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.hpp"
#include "mlp.hpp"

extern "C" {
#include "adatm_b200.h"
}

using namespace adatm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *msg) {
  g_last_error = msg;
  return code;
}

template <typename F>
int guarded(F &&f) {
  g_last_error.clear();
  try {
    f();
    return SPLATT_SUCCESS;
  } catch (const BadInput &e) {
    return fail(SPLATT_ERROR_BADINPUT, e.what());
  } catch (const NoMemory &e) {
    return fail(SPLATT_ERROR_NOMEMORY, e.what());
  } catch (const CudaError &e) {
    return fail(ADATM_ERROR_CUDA, e.what());
  } catch (const std::bad_alloc &e) {
    return fail(SPLATT_ERROR_NOMEMORY, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(SPLATT_ERROR_BADINPUT, e.what());
  }
}

cudaStream_t new_stream() {
  cudaStream_t s;
  ADATM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

struct StreamOwner {
  cudaStream_t s = nullptr;
  StreamOwner() : s(new_stream()) {}
  ~StreamOwner() {
    if (s) cudaStreamDestroy(s);
  }
};

// Device state behind a host splatt_csf array.
struct CsfHandle {
  StreamOwner stream;
  std::shared_ptr<DevCoo> coo;
  std::vector<std::shared_ptr<DevCsf>> trees;
  Plan plan;
  splatt_csf *host = nullptr;
  int n_csf = 0;
  // engines by rank and group list (a caller may pass other memo levels
  // for the same trees); each keeps its own factors and memo rows
  std::map<std::string, std::unique_ptr<Engine>> engines;
  std::vector<rcsf_seq_adaptive *> memo_views;
  // the handle's own plan, with its own trees and tags per mode
  Engine &engine(uint64_t R) {
    Engine &e = engine(R, plan);
    e.set_use(plan.use_csfs, plan.use_tags);
    return e;
  }
  Engine &engine(uint64_t R, const Plan &p) {
    std::string key = std::to_string(R) + (p.space_efficient ? "s" : "t");
    for (int g = 0; g < p.n_grp; ++g) {
      key += "|" + std::to_string(p.grp[g].memo_mode) + "," + std::to_string(p.grp[g].begin_imten) +
             "," + std::to_string(p.grp[g].n_imten) + ":";
      for (int l = 0; l < p.nmodes; ++l) key += std::to_string(p.grp[g].o_opt[l]) + ".";
    }
    auto it = engines.find(key);
    if (it != engines.end()) return *it->second;
    EngineOptions o;
    auto e = std::make_unique<Engine>(coo, trees, R, p, o, stream.s);
    Engine &ref = *e;
    engines[key] = std::move(e);
    return ref;
  }
};

std::mutex g_mu;
std::unordered_map<const void *, std::shared_ptr<CsfHandle>> g_csf;      // by splatt_csf array
std::unordered_map<const void *, std::shared_ptr<CsfHandle>> g_rcsf;     // by rcsf_seq array

std::shared_ptr<CsfHandle> find_csf(const void *p) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_csf.find(p);
  if (it == g_csf.end()) throw BadInput("these trees were not built by this library");
  return it->second;
}

uint64_t *host_u64(size_t n) {
  uint64_t *p = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
  if (!p) throw std::bad_alloc();
  return p;
}

// Fill the host splatt_csf array (reference layout: fids[0] == NULL, one
// tile) from the device trees.
void fill_host_trees(CsfHandle &h, const uint64_t *dims) {
  const int N = h.coo->nmodes;
  h.host = (splatt_csf *)calloc(h.trees.size(), sizeof(splatt_csf));
  if (!h.host) throw std::bad_alloc();
  h.n_csf = (int)h.trees.size();
  for (size_t g = 0; g < h.trees.size(); ++g) {
    const DevCsf &c = *h.trees[g];
    splatt_csf &o = h.host[g];
    o.nnz = c.nnz;
    o.nmodes = (splatt_idx_t)N;
    for (int m = 0; m < N; ++m) {
      o.dims[m] = dims[m];
      o.dim_perm[m] = c.dim_perm[m];
      o.tile_dims[m] = 1;
    }
    o.which_tile = SPLATT_NOTILE;
    o.ntiles = 1;
    o.pt = (csf_sparsity *)calloc(1, sizeof(csf_sparsity));
    HostCsfArrays a;
    csf_download(c, a, h.stream.s);
    for (int l = 0; l < N; ++l) {
      o.pt->nfibs[l] = c.nfibs[l];
      if (l < N - 1) {
        o.pt->fptr[l] = host_u64(a.fptr[l].size());
        memcpy(o.pt->fptr[l], a.fptr[l].data(), a.fptr[l].size() * sizeof(uint64_t));
      }
      if (l >= 1) {
        o.pt->fids[l] = host_u64(a.fids[l].size());
        memcpy(o.pt->fids[l], a.fids[l].data(), a.fids[l].size() * sizeof(uint64_t));
      }
    }
    o.pt->vals = (double *)malloc((c.nnz ? c.nnz : 1) * sizeof(double));
    memcpy(o.pt->vals, a.vals.data(), c.nnz * sizeof(double));
  }
}

void free_host_trees(splatt_csf *t, int n) {
  if (!t) return;
  for (int g = 0; g < n; ++g) {
    if (!t[g].pt) continue;
    for (int l = 0; l < (int)t[g].nmodes; ++l) {
      free(t[g].pt->fptr[l]);
      free(t[g].pt->fids[l]);
    }
    free(t[g].pt->vals);
    free(t[g].pt);
  }
  free(t);
}

std::shared_ptr<DevCoo> upload_coo(int N, uint64_t nnz, const uint64_t *dims,
                                   const uint64_t *const *inds, const double *vals,
                                   cudaStream_t s) {
  auto c = std::make_shared<DevCoo>();
  coo_upload(*c, N, nnz, dims, inds, vals, s);
  return c;
}

std::shared_ptr<CsfHandle> make_handle(std::shared_ptr<DevCoo> coo, const Plan &plan) {
  auto h = std::make_shared<CsfHandle>();
  h->coo = std::move(coo);
  h->plan = plan;
  for (int g = 0; g < plan.n_csf; ++g) {
    h->trees.push_back(std::make_shared<DevCsf>());
    csf_build(*h->coo, plan.tree(g).o_opt, *h->trees.back(), h->stream.s);
  }
  fill_host_trees(*h, h->coo->dims);
  std::lock_guard<std::mutex> lk(g_mu);
  g_csf[h->host] = h;
  return h;
}

Plan plan_from_groups(int N, const group_properties *grp, idx_t n_grp, bool space = false) {
  Plan p;
  p.nmodes = N;
  p.n_grp = (int)n_grp;
  for (idx_t g = 0; g < n_grp; ++g) {
    p.grp[g].memo_mode = grp[g].memo_mode;
    p.grp[g].begin_imten = grp[g].begin_imten;
    p.grp[g].n_imten = grp[g].n_imten;
    for (int m = 0; m < N; ++m) p.grp[g].o_opt[m] = grp[g].o_opt[m];
  }
  if (space) decide_use_csfs_space(p);
  else decide_use_csfs(p);
  return p;
}

void check_plan(const Plan &p) {
  const int N = p.nmodes;
  if (p.n_grp < 1 || p.n_grp > N) throw BadInput("bad group count");
  for (int g = 0; g < p.n_grp; ++g) {
    bool seen[kMaxModes] = {false};
    for (int l = 0; l < N; ++l) {
      if (p.grp[g].o_opt[l] >= (uint64_t)N || seen[p.grp[g].o_opt[l]])
        throw BadInput("o_opt is not a permutation of the modes");
      seen[p.grp[g].o_opt[l]] = true;
    }
    if (p.grp[g].n_imten > 0 &&
        (p.grp[g].begin_imten > (uint64_t)N - 1 || p.grp[g].n_imten > p.grp[g].begin_imten))
      throw BadInput("memo levels outside the tree");
  }
}


// The group list a reference caller passes with a call (grp_prop, n_grp and
// n_csf, as csf_alloc_adaptive / decide_use_csfs read them), checked against
// the trees the handle holds: the same number of trees, each in the level
// order its group names. The memo levels (begin_imten, n_imten) may differ
// from the handle's: they select the engine. With grp == nullptr the
// handle's own plan. The memo sequences rs_seq (when given) must describe
// the same memo levels as the groups.
Plan caller_plan(const CsfHandle &h, const group_properties *grp, idx_t n_grp, idx_t n_csf,
                 const rcsf_seq_adaptive *rs_seq) {
  const int N = h.coo->nmodes;
  if (n_csf != (idx_t)h.plan.n_csf)
    throw BadInput("n_csf (" + std::to_string(n_csf) + ") is not the number of trees built (" +
                   std::to_string(h.plan.n_csf) + ")");
  Plan p = h.plan;
  if (grp != nullptr) {
    if (n_grp < 1 || n_grp > (idx_t)N) throw BadInput("n_grp out of range");
    for (idx_t g = 0; g < n_grp; ++g)
      if (grp[g].o_opt == nullptr) throw BadInput("grp_prop has a group without o_opt");
    p = plan_from_groups(N, grp, n_grp, n_csf != n_grp);
    check_plan(p);
    if (p.n_csf != h.plan.n_csf)
      throw BadInput("grp_prop describes a different number of trees than were built");
    for (int t = 0; t < p.n_csf; ++t)
      for (int l = 0; l < N; ++l)
        if (p.tree(t).o_opt[l] != h.trees[t]->dim_perm[l])
          throw BadInput("grp_prop's o_opt is not the level order of the trees these were built with");
  }
  if (rs_seq != nullptr) {
    idx_t j = 0;
    for (int t = 0; t < p.n_csf; ++t) {
      const Group &gp = p.tree(t);
      if (gp.n_imten == 0) continue;
      if (rs_seq[j].begin_imten != gp.begin_imten || rs_seq[j].n_imten != gp.n_imten)
        throw BadInput("rs_seq's memo levels differ from grp_prop's");
      ++j;
    }
  }
  return p;
}

// The engine of a reference caller's ALS call: its groups (memo levels) and
// its per-mode trees and tags (use_csfs / use_tags, validated by set_use).
Engine &caller_engine(CsfHandle &h, rcsf_seq_adaptive const *rs_seq, idx_t n_csf,
                      group_properties const *grp_prop, idx_t n_grp, idx_t const *use_csfs,
                      idx_t const *use_tags, uint64_t R) {
  const Plan p = caller_plan(h, grp_prop, grp_prop ? n_grp : 0, n_csf, rs_seq);
  Engine &e = h.engine(R, p);
  if ((use_csfs == nullptr) != (use_tags == nullptr))
    throw BadInput("use_csfs and use_tags must be given together");
  if (use_csfs != nullptr) {
    uint64_t uc[kMaxModes], ut[kMaxModes];
    for (int m = 0; m < e.nmodes(); ++m) {
      uc[m] = use_csfs[m];
      ut[m] = use_tags[m];
    }
    e.set_use(uc, ut);
  } else {
    e.set_use(p.use_csfs, p.use_tags);
  }
  return e;
}

// The ALS loop shared by the splatt_* entry points, with the reference's
// per-iteration report (adatm_cpd.c:343-354).
// With `out`, the last iteration's factors come back normalised into `out`
// and `lambda` while that sweep runs (Engine::sweep_download) and
// *downloaded is set; a tolerance stop before it leaves them on the device.
double run_als(Engine &e, uint64_t niters, double tol, int verbosity, double *const *out = nullptr,
               double *lambda = nullptr, bool *downloaded = nullptr) {
  e.als_begin();
  e.capture_graph();  // one sweep as a CUDA graph, reused across calls
  double fit = 0, old = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (uint64_t it = 0; it < niters; ++it) {
    const auto ti = std::chrono::steady_clock::now();
    if (out != nullptr && it + 1 == niters) {
      fit = e.sweep_download(out, lambda);
      *downloaded = true;
    } else {
      e.sweep();
      fit = e.fit_host();
    }
    if (verbosity > SPLATT_VERBOSITY_NONE) {
      const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - ti).count();
      printf("  its = %3" PRIu64 " (%0.3fs)  fit = %0.5f  delta = %+0.4e\n", it + 1, s, fit,
             fit - old);
    }
    if (it > 0 && std::fabs(fit - old) < tol) break;
    old = fit;
  }
  if (verbosity > SPLATT_VERBOSITY_NONE)
    printf("CPD = %0.3fs\n",
           std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  return fit;
}

void fill_kruskal(Engine &e, double fit, splatt_kruskal *k) {
  const int N = e.nmodes();
  const uint64_t R = e.rank();
  k->rank = R;
  k->nmodes = (splatt_idx_t)N;
  k->fit = fit;
  k->lambda = (double *)malloc(R * sizeof(double));
  double *mats[kMaxModes];
  for (int m = 0; m < N; ++m) {
    k->dims[m] = e.dims()[m];
    k->factors[m] = (double *)malloc((size_t)e.dims()[m] * R * sizeof(double));
    mats[m] = k->factors[m];
  }
  e.get_normalized(mats, k->lambda);
}

void plan_to_c(const Plan &p, adatm_plan *o) {
  memset(o, 0, sizeof(*o));
  o->nmodes = p.nmodes;
  o->n_grp = p.n_grp;
  for (int g = 0; g < p.n_grp; ++g) {
    o->memo_mode[g] = p.grp[g].memo_mode;
    o->begin_imten[g] = p.grp[g].begin_imten;
    o->n_imten[g] = p.grp[g].n_imten;
    for (int l = 0; l < p.nmodes; ++l) o->o_opt[g][l] = p.grp[g].o_opt[l];
  }
  o->space_efficient = p.space_efficient ? 1 : 0;
  for (int m = 0; m < p.nmodes; ++m) {
    o->use_csfs[m] = p.use_csfs[m];
    o->use_tags[m] = p.use_tags[m];
  }
}

Plan plan_from_c(const adatm_plan *c) {
  Plan p;
  p.nmodes = c->nmodes;
  p.n_grp = c->n_grp;
  for (int g = 0; g < c->n_grp; ++g) {
    p.grp[g].memo_mode = c->memo_mode[g];
    p.grp[g].begin_imten = c->begin_imten[g];
    p.grp[g].n_imten = c->n_imten[g];
    for (int l = 0; l < c->nmodes; ++l) p.grp[g].o_opt[l] = c->o_opt[g][l];
  }
  for (int m = 0; m < c->nmodes; ++m) {
    p.use_csfs[m] = c->use_csfs[m];
    p.use_tags[m] = c->use_tags[m];
  }
  p.n_csf = p.n_grp;
  if (c->space_efficient) decide_use_csfs_space(p);
  return p;
}

int adatm_engine_memo_raw(Engine *g, int grp, int deg, double *out);

std::shared_ptr<DevCoo> coo_of(sptensor_t *tt, cudaStream_t s) {
  return upload_coo((int)tt->nmodes, tt->nnz, tt->dims, tt->ind, tt->vals, s);
}

template <typename T>
void pull_rows(Engine &e, const T *src, uint64_t rows, double *out) {
  const int ldr = e.ldr();
  const uint64_t R = e.rank();
  std::vector<T> buf((size_t)rows * ldr);
  if (rows)
    ADATM_CUDA(cudaMemcpyAsync(buf.data(), src, buf.size() * sizeof(T), cudaMemcpyDeviceToHost,
                               e.stream()));
  ADATM_CUDA(cudaStreamSynchronize(e.stream()));
  for (uint64_t i = 0; i < rows; ++i)
    for (uint64_t r = 0; r < R; ++r) out[i * R + r] = buf[i * ldr + r];
}

}  // namespace

// ===========================================================================
// adatm_tensor / adatm_engine
// ===========================================================================
struct adatm_tensor {
  StreamOwner stream;
  std::shared_ptr<DevCoo> coo;
};

struct adatm_batch {
  StreamOwner stream;
  std::unique_ptr<BatchSweep> batch;
};

struct adatm_mlp {
  StreamOwner stream;
  std::unique_ptr<Mlp> net;
};

struct adatm_engine {
  StreamOwner stream;
  std::unique_ptr<Engine> eng;
  bool graph = false;
};

extern "C" {

const char *adatm_last_error(void) { return g_last_error.c_str(); }

int adatm_set_device(int device) {
  return guarded([&] { ADATM_CUDA(cudaSetDevice(device)); });
}

// ---------------------------------------------------------------------------
// options
// ---------------------------------------------------------------------------
double *splatt_default_opts(void) {
  double *o = (double *)calloc(SPLATT_OPTION_NOPTIONS, sizeof(double));
  if (!o) return nullptr;
  o[SPLATT_OPTION_NTHREADS] = 1;
  o[SPLATT_OPTION_TOLERANCE] = 1e-5;
  o[SPLATT_OPTION_NITER] = 50;
  o[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  o[SPLATT_OPTION_RANDSEED] = 0;
  o[SPLATT_OPTION_CSF_ALLOC] = SPLATT_ADAPTIVE_TIME_EFFICIENT;
  o[SPLATT_OPTION_TILE] = SPLATT_NOTILE;
  o[SPLATT_OPTION_TILEDEPTH] = 1;
  o[SPLATT_OPTION_DECOMP] = SPLATT_DECOMP_MEDIUM;
  o[SPLATT_OPTION_COMM] = SPLATT_COMM_ALL2ALL;
  return o;
}

void splatt_free_opts(double *opts) { free(opts); }

// ---------------------------------------------------------------------------
// SPLATT public data structures
// ---------------------------------------------------------------------------
int splatt_csf_convert(splatt_idx_t const nmodes, splatt_idx_t const nnz,
                       splatt_idx_t **const inds, splatt_val_t *const vals,
                       splatt_csf **tensors, double const *const options) {
  return guarded([&] {
    if (!inds || !vals || !tensors) throw BadInput("null argument");
    if ((int)options[SPLATT_OPTION_TILE] != SPLATT_NOTILE) throw BadInput("only SPLATT_NOTILE is supported");
    std::vector<uint64_t> dims(nmodes, 0);
    for (idx_t m = 0; m < nmodes; ++m)
      for (idx_t n = 0; n < nnz; ++n) dims[m] = std::max(dims[m], inds[m][n] + 1);
    StreamOwner tmp;
    auto coo = upload_coo((int)nmodes, nnz, dims.data(), inds, vals, tmp.s);
    const int alloc = (int)options[SPLATT_OPTION_CSF_ALLOC];
    Plan p;
    if (alloc <= SPLATT_CSF_ALLMODE) {
      p = plan_splatt((int)nmodes, dims.data(), alloc);
    } else {
      p = plan_analytic(*coo, 16, 1, nullptr, tmp.s);
    }
    auto h = make_handle(coo, p);
    *tensors = h->host;
  });
}

int splatt_csf_load(char const *const fname, splatt_idx_t *nmodes, splatt_csf **tensors,
                    double const *const options) {
  std::vector<std::vector<uint64_t>> ind;
  std::vector<double> val;
  int rc = guarded([&] {
    FILE *f = fopen(fname, "r");
    if (!f) throw BadInput("cannot open tensor file");
    char line[4096];
    int N = 0;
    while (fgets(line, sizeof(line), f)) {
      if (line[0] == '#' || line[0] == '\n' || line[0] == '\0') continue;
      std::vector<double> tok;
      char *p = line;
      while (*p) {
        char *end;
        const double v = strtod(p, &end);
        if (end == p) break;
        tok.push_back(v);
        p = end;
      }
      if (tok.size() < 2) continue;
      if (N == 0) {
        N = (int)tok.size() - 1;
        ind.assign(N, {});
      }
      if ((int)tok.size() != N + 1) {
        fclose(f);
        throw BadInput("inconsistent number of modes in tensor file");
      }
      for (int m = 0; m < N; ++m) {
        if (tok[m] < 1) {
          fclose(f);
          throw BadInput("tensor file indices are 1-based");
        }
        ind[m].push_back((uint64_t)tok[m] - 1);
      }
      val.push_back(tok[N]);
    }
    fclose(f);
    if (N == 0) throw BadInput("empty tensor file");
    *nmodes = (splatt_idx_t)N;
  });
  if (rc != SPLATT_SUCCESS) return rc;
  std::vector<splatt_idx_t *> ptrs(ind.size());
  for (size_t m = 0; m < ind.size(); ++m) ptrs[m] = ind[m].data();
  return splatt_csf_convert(*nmodes, val.size(), ptrs.data(), val.data(), tensors, options);
}

void splatt_free_csf(splatt_csf *tensors, double const *const options) {
  (void)options;
  if (!tensors) return;
  std::shared_ptr<CsfHandle> h;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_csf.find(tensors);
    if (it != g_csf.end()) {
      h = it->second;
      g_csf.erase(it);
    }
    for (auto it2 = g_rcsf.begin(); it2 != g_rcsf.end();)
      if (it2->second == h) it2 = g_rcsf.erase(it2);
      else ++it2;
  }
  if (h) {
    free_host_trees(h->host, h->n_csf);
    h->host = nullptr;
  }
}

void splatt_free_kruskal(splatt_kruskal *factored) {
  if (!factored) return;
  free(factored->lambda);
  for (idx_t m = 0; m < factored->nmodes; ++m) free(factored->factors[m]);
}

int splatt_cpd_als(splatt_csf const *const tensors, splatt_idx_t const nfactors,
                   double const *const options, splatt_kruskal *factored) {
  return guarded([&] {
    auto h = find_csf(tensors);
    Engine &e = h->engine(nfactors);
    e.init_factors((uint64_t)options[SPLATT_OPTION_RANDSEED]);
    const double fit = run_als(e, (uint64_t)options[SPLATT_OPTION_NITER],
                               options[SPLATT_OPTION_TOLERANCE],
                               (int)options[SPLATT_OPTION_VERBOSITY]);
    fill_kruskal(e, fit, factored);
  });
}

int splatt_mttkrp(splatt_idx_t const mode, splatt_idx_t const ncolumns,
                  splatt_csf const *const tensors, splatt_val_t **matrices,
                  splatt_val_t *const matout, double const *const options) {
  (void)options;
  return guarded([&] {
    auto h = find_csf(tensors);
    if (mode >= (idx_t)h->coo->nmodes) throw BadInput("mode out of range");
    Engine &e = h->engine(ncolumns);
    e.set_factors(matrices);
    e.mttkrp_direct((int)mode, e.mttkrp_buffer());
    const uint64_t I = e.dims()[mode];
    std::vector<double> buf((size_t)I * e.ldr());
    ADATM_CUDA(cudaMemcpyAsync(buf.data(), e.mttkrp_buffer(), buf.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, e.stream()));
    ADATM_CUDA(cudaStreamSynchronize(e.stream()));
    for (uint64_t i = 0; i < I; ++i)
      for (uint64_t r = 0; r < ncolumns; ++r) matout[i * ncolumns + r] = buf[i * e.ldr() + r];
  });
}

// ---------------------------------------------------------------------------
// AdaTM entry points
// ---------------------------------------------------------------------------
void decide_product_order(sptensor_t *const tt, idx_t **product_order) {
  const idx_t N = tt->nmodes;
  for (idx_t m = 0; m < N; ++m) {
    memset(product_order[m], 0, 2 * N * sizeof(idx_t));
    for (idx_t i = m + 1; i < N; ++i) product_order[m][i] = 1;
    for (idx_t i = 0; i < m; ++i) product_order[m][i + N] = 1;
  }
}

static group_properties *groups_to_c(const Plan &p) {
  group_properties *g = (group_properties *)calloc(p.n_grp, sizeof(group_properties));
  for (int i = 0; i < p.n_grp; ++i) {
    g[i].memo_mode = p.grp[i].memo_mode;
    g[i].begin_imten = p.grp[i].begin_imten;
    g[i].n_imten = p.grp[i].n_imten;
    g[i].o_opt = (idx_t *)malloc(p.nmodes * sizeof(idx_t));
    for (int l = 0; l < p.nmodes; ++l) g[i].o_opt[l] = p.grp[i].o_opt[l];
  }
  return g;
}

idx_t decide_parameters_auto(sptensor_t *const tt, idx_t const nfactors, int strategy,
                             idx_t const **product_order, group_properties **grp_prop) {
  (void)product_order;
  idx_t n = 0;
  int rc = guarded([&] {
    StreamOwner s;
    auto coo = coo_of(tt, s.s);
    Plan p = plan_analytic(*coo, nfactors, strategy, nullptr, s.s);
    *grp_prop = groups_to_c(p);
    n = (idx_t)p.n_grp;
  });
  if (rc != SPLATT_SUCCESS) {
    fprintf(stderr, "decide_parameters_auto: %s\n", g_last_error.c_str());
    *grp_prop = nullptr;
    return 0;
  }
  return n;
}

idx_t decide_candidate_configs(sptensor_t *const tt, idx_t const **product_order,
                               configurations_adaptive **configs) {
  (void)product_order;
  std::vector<Candidate> c = candidate_configs((int)tt->nmodes, tt->dims);
  *configs = (configurations_adaptive *)calloc(c.size() ? c.size() : 1, sizeof(configurations_adaptive));
  for (size_t i = 0; i < c.size(); ++i) {
    (*configs)[i].n_grp = (idx_t)c[i].plan.n_grp;
    (*configs)[i].grp_prop = groups_to_c(c[i].plan);
  }
  return (idx_t)c.size();
}

void predict_candidates_adaptive(sptensor_t *const tt, idx_t const nfactors,
                                 configurations_adaptive *configs, idx_t const nconfigs) {
  int rc = guarded([&] {
    StreamOwner s;
    auto coo = coo_of(tt, s.s);
    std::vector<Candidate> c(nconfigs);
    for (idx_t i = 0; i < nconfigs; ++i)
      c[i].plan = plan_from_groups((int)tt->nmodes, configs[i].grp_prop, configs[i].n_grp);
    predict_candidates(*coo, nfactors, c, s.s);
    for (idx_t i = 0; i < nconfigs; ++i) {
      configs[i].pspace = c[i].pspace;
      configs[i].pops = c[i].pops;
    }
  });
  if (rc != SPLATT_SUCCESS) fprintf(stderr, "predict_candidates_adaptive: %s\n", g_last_error.c_str());
}

idx_t limit_candidates_by_space(configurations_adaptive const *const configs,
                                idx_t const nconfigs, idx_t **const real_config_locs) {
  idx_t n = 0;
  for (idx_t c = 0; c < nconfigs; ++c)
    if ((double)configs[c].pspace < 90e9) ++n;
  *real_config_locs = (idx_t *)malloc((n ? n : 1) * sizeof(idx_t));
  n = 0;
  for (idx_t c = 0; c < nconfigs; ++c)
    if ((double)configs[c].pspace < 90e9) (*real_config_locs)[n++] = c;
  return n;
}

idx_t choose_candidates_by_strategy(configurations_adaptive const *const configs,
                                    idx_t const nconfigs, idx_t const *const real_config_locs,
                                    idx_t const n_real_configs, int strategy) {
  (void)nconfigs;
  idx_t best = 0;
  for (idx_t c = 1; c < n_real_configs; ++c) {
    const configurations_adaptive &x = configs[real_config_locs[c]];
    const configurations_adaptive &b = configs[real_config_locs[best]];
    if (strategy == 2 ? x.pspace < b.pspace : x.pops < b.pops) best = c;
  }
  return best;
}

splatt_csf *csf_alloc_adaptive(sptensor_t *const tt, group_properties *const grp_prop,
                               idx_t const n_grp, double const *const opts, idx_t *n_csf) {
  splatt_csf *out = nullptr;
  int rc = guarded([&] {
    (void)opts;
    StreamOwner s;
    auto coo = coo_of(tt, s.s);
    const bool space =
        opts != nullptr && (int)opts[SPLATT_OPTION_CSF_ALLOC] == SPLATT_ADAPTIVE_SPACE_EFFICIENT;
    Plan p = plan_from_groups((int)tt->nmodes, grp_prop, n_grp, space);
    check_plan(p);
    auto h = make_handle(coo, p);
    *n_csf = (idx_t)h->n_csf;
    out = h->host;
  });
  if (rc != SPLATT_SUCCESS) fprintf(stderr, "csf_alloc_adaptive: %s\n", g_last_error.c_str());
  return out;
}

rcsf_seq_adaptive *rcsf_alloc_adaptive(splatt_csf *const ct, idx_t const nfactors,
                                       group_properties *const grp_prop, idx_t const n_grp,
                                       idx_t const n_csf, double const *const opts,
                                       idx_t *n_rcsf) {
  (void)opts;
  (void)n_csf;
  rcsf_seq_adaptive *ret = nullptr;
  int rc = guarded([&] {
    auto h = find_csf(ct);
    h->engine(nfactors);  // memo rows in HBM
    (void)grp_prop;
    (void)n_grp;
    const Plan &plan = h->plan;
    ret = (rcsf_seq_adaptive *)calloc(plan.n_csf ? plan.n_csf : 1, sizeof(rcsf_seq_adaptive));
    idx_t j = 0;
    for (int t = 0; t < plan.n_csf; ++t) {  // one memo sequence per memoizing tree
      const Group &gp = plan.tree(t);
      if (gp.n_imten == 0) continue;
      rcsf_seq_adaptive &sq = ret[j++];
      sq.begin_imten = gp.begin_imten;
      sq.n_imten = gp.n_imten;
      sq.rcsfs = (splatt_csf *)calloc(sq.n_imten, sizeof(splatt_csf));
      const splatt_csf &c = ct[t];
      // memo tree layout of p_rcsf_alloc_untiled_adaptive (adatm_rcsf.c:216-278)
      for (idx_t deg = 0; deg < sq.n_imten; ++deg) {
        splatt_csf &o = sq.rcsfs[deg];
        const idx_t nm = sq.begin_imten - deg + 1;
        o.nmodes = nm;
        for (idx_t m = 0; m < nm; ++m) {
          o.dims[m] = c.dims[c.dim_perm[m]];
          o.dim_perm[m] = c.dim_perm[m];
          o.tile_dims[m] = 1;
        }
        o.dims[nm - 1] = nfactors;
        o.which_tile = SPLATT_NOTILE;
        o.ntiles = 1;
        o.nnz = c.pt->nfibs[nm - 2] * nfactors;
        o.pt = (csf_sparsity *)calloc(1, sizeof(csf_sparsity));
        for (idx_t m = 0; m + 1 < nm; ++m) o.pt->nfibs[m] = c.pt->nfibs[m];
        o.pt->nfibs[nm - 1] = o.nnz;
        for (idx_t m = 0; m + 2 < nm; ++m) {
          o.pt->fptr[m] = c.pt->fptr[m];
          o.pt->fids[m] = c.pt->fids[m];
        }
        o.pt->fids[nm - 2] = c.pt->fids[nm - 2];
        o.pt->vals = (double *)calloc(o.nnz ? o.nnz : 1, sizeof(double));
      }
    }
    *n_rcsf = j;
    h->memo_views.push_back(ret);
    std::lock_guard<std::mutex> lk(g_mu);
    g_rcsf[ret] = h;
  });
  if (rc != SPLATT_SUCCESS) fprintf(stderr, "rcsf_alloc_adaptive: %s\n", g_last_error.c_str());
  return ret;
}

size_t csf_storage_adaptive(splatt_csf const *const tensors, idx_t const n_csf,
                            group_properties *const grp_prop, int const n_grp) {
  (void)grp_prop;
  (void)n_grp;
  size_t bytes = 0;  // adatm_rcsf.c:562-588
  for (idx_t g = 0; g < n_csf; ++g) {
    const splatt_csf &c = tensors[g];
    bytes += c.nnz * sizeof(val_t) + c.nnz * sizeof(idx_t) + c.ntiles * sizeof(csf_sparsity);
    for (idx_t m = 0; m + 1 < c.nmodes; ++m) {
      bytes += (c.pt->nfibs[m] + 1) * sizeof(idx_t);
      if (c.pt->fids[m] != nullptr) bytes += c.pt->nfibs[m] * sizeof(idx_t);
    }
  }
  return bytes;
}

size_t rcsf_storage_adaptive(rcsf_seq_adaptive const *const seq_rcsf, idx_t const n_csf) {
  size_t bytes = 0;  // adatm_rcsf.c:618-638
  for (idx_t j = 0; j < n_csf; ++j)
    for (idx_t d = 0; d < seq_rcsf[j].n_imten; ++d)
      bytes += seq_rcsf[j].rcsfs[d].nnz * sizeof(val_t) + sizeof(csf_sparsity);
  return bytes;
}

void decide_use_csfs(idx_t const nmodes, group_properties *const grp_prop, int const n_grp,
                     idx_t const n_csf, idx_t *use_csfs, idx_t *use_tags) {
  // the reference takes the SPACE_EFFICIENT branch when fewer trees than
  // groups were built (mttkrp.c:1976)
  Plan p = plan_from_groups((int)nmodes, grp_prop, (idx_t)n_grp, n_csf != (idx_t)n_grp);
  for (idx_t m = 0; m < nmodes; ++m) {
    use_csfs[m] = p.use_csfs[m];
    use_tags[m] = p.use_tags[m];
  }
}

void mttkrp_csf_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive const *const rs_seq,
                         idx_t const n_csf, matrix_t **mats, idx_t const mode,
                         thd_info *const thds, group_properties *const grp_prop,
                         int const n_grp, idx_t const use_csf, idx_t const use_tag,
                         double const *const opts) {
  (void)thds;
  (void)opts;
  int rc = guarded([&] {
    auto h = find_csf(tensors);
    const int N = h->coo->nmodes;
    if (mode >= (idx_t)N) throw BadInput("mode out of range");
    const uint64_t R = mats[0]->J;
    // the caller's groups pick the engine (memo levels); its tree and tag
    // pick the walk, as the reference's dispatch does (mttkrp.c:2058-2087)
    const Plan p = caller_plan(*h, grp_prop, grp_prop ? (idx_t)n_grp : 0, n_csf, rs_seq);
    Engine &e = h->engine(R, p);
    e.check_use((int)mode, (int)std::min<idx_t>(use_csf, kMaxModes), (int)std::min<idx_t>(use_tag, 3));
    const double *fm[kMaxModes];
    for (int m = 0; m < N; ++m) fm[m] = mats[m]->vals;
    e.set_factors(fm);
    e.mttkrp_with((int)mode, (int)use_csf, (int)use_tag, e.mttkrp_buffer());
    const uint64_t I = e.dims()[mode];
    std::vector<double> buf((size_t)I * e.ldr());
    ADATM_CUDA(cudaMemcpyAsync(buf.data(), e.mttkrp_buffer(), buf.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, e.stream()));
    ADATM_CUDA(cudaStreamSynchronize(e.stream()));
    matrix_t *M = mats[SPLATT_MAX_NMODES];
    M->I = I;
    for (uint64_t i = 0; i < I; ++i)
      for (uint64_t r = 0; r < R; ++r) M->vals[i * R + r] = buf[i * e.ldr() + r];
  });
  if (rc != SPLATT_SUCCESS) fprintf(stderr, "mttkrp_csf_adaptive: %s\n", g_last_error.c_str());
}

double cpd_als_iterate_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive *const rs_seq,
                                splatt_idx_t const n_csf, group_properties const *const grp_prop,
                                splatt_idx_t const n_grp, splatt_idx_t const *const use_csfs,
                                splatt_idx_t const *const use_tags, matrix_t **mats,
                                val_t *const lambda, idx_t const nfactors,
                                rank_info *const rinfo, double const *const opts) {
  (void)rinfo;
  double fit = 0;
  int rc = guarded([&] {
    auto h = find_csf(tensors);
    const int N = h->coo->nmodes;
    Engine &e = caller_engine(*h, rs_seq, n_csf, grp_prop, n_grp, use_csfs, use_tags, nfactors);
    const double *fm[kMaxModes];
    double *om[kMaxModes];
    for (int m = 0; m < N; ++m) {
      fm[m] = mats[m]->vals;
      om[m] = mats[m]->vals;
    }
    e.set_factors(fm);
    bool downloaded = false;
    fit = run_als(e, (uint64_t)opts[SPLATT_OPTION_NITER], opts[SPLATT_OPTION_TOLERANCE],
                  (int)opts[SPLATT_OPTION_VERBOSITY], om, lambda, &downloaded);
    if (!downloaded) e.get_normalized(om, lambda);
  });
  if (rc != SPLATT_SUCCESS) {
    fprintf(stderr, "cpd_als_iterate_adaptive: %s\n", g_last_error.c_str());
    fit = std::nan("");
  }
  return fit;
}

int splatt_cpd_als_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive *const rs_seq,
                            splatt_idx_t const n_csf, group_properties const *const grp_prop,
                            splatt_idx_t const n_grp, splatt_idx_t const *const use_csfs,
                            splatt_idx_t const *const use_tags, splatt_idx_t const nfactors,
                            double const *const options, splatt_kruskal *factored) {
  return guarded([&] {
    auto h = find_csf(tensors);
    Engine &e = caller_engine(*h, rs_seq, n_csf, grp_prop, n_grp, use_csfs, use_tags, nfactors);
    e.init_factors((uint64_t)options[SPLATT_OPTION_RANDSEED]);
    const double fit = run_als(e, (uint64_t)options[SPLATT_OPTION_NITER],
                               options[SPLATT_OPTION_TOLERANCE],
                               (int)options[SPLATT_OPTION_VERBOSITY]);
    fill_kruskal(e, fit, factored);
  });
}

void bench_adaptm(sptensor_t *const tt, matrix_t **mats, bench_opts const *const opts) {
  int rc = guarded([&] {
    StreamOwner s;
    auto coo = coo_of(tt, s.s);
    const uint64_t R = mats[0]->J;
    Plan p = plan_analytic(*coo, R, 1, nullptr, s.s);
    printf("Optimal predicted group properties:\nNumber of groups: %d\n", p.n_grp);
    {
      group_properties *gp = groups_to_c(p);
      char title[] = "Optimal grp_prop";
      print_group_properties(gp, (idx_t)p.n_grp, (idx_t)p.nmodes, title);
      adatm_free_groups(gp, (idx_t)p.n_grp);
    }
    EngineOptions eo;
    Engine e(coo, {}, R, p, eo, s.s);
    printf("Number of CSFs: %d\nCSF-STORAGE: %zu B\nvCSF-STORAGE: %zu B\n", e.n_csf(),
           e.csf_bytes(), e.memo_bytes());
    const double *fm[kMaxModes];
    for (int m = 0; m < (int)tt->nmodes; ++m) fm[m] = mats[m]->vals;
    e.set_factors(fm);
    cudaEvent_t a, b;
    ADATM_CUDA(cudaEventCreate(&a));
    ADATM_CUDA(cudaEventCreate(&b));
    for (idx_t i = 0; i < opts->niters; ++i) {
      double its = 0;
      for (int m = 0; m < (int)tt->nmodes; ++m) {
        ADATM_CUDA(cudaEventRecord(a, s.s));
        e.mttkrp(m, e.mttkrp_buffer());
        ADATM_CUDA(cudaEventRecord(b, s.s));
        ADATM_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        ADATM_CUDA(cudaEventElapsedTime(&ms, a, b));
        its += ms / 1e3;
        printf("  mode %d %0.3fs\n", m + 1, ms / 1e3);
      }
      printf("    its = %3" PRIu64 " (%0.3fs)\n", i + 1, its);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
  if (rc != SPLATT_SUCCESS) fprintf(stderr, "bench_adaptm: %s\n", g_last_error.c_str());
}

static void stats_one(splatt_csf const *ct) {
  // p_stats_csf_mode (adatm_stats.c:19-49): one tile, never empty here
  printf("nmodes: %" PRIu64 " nnz: %" PRIu64 "\n", ct->nmodes, ct->nnz);
  printf("dims: %" PRIu64 "", ct->dims[0]);
  for (idx_t m = 1; m < ct->nmodes; ++m) printf("x%" PRIu64 "", ct->dims[m]);
  printf(" (%" PRIu64 "", ct->dim_perm[0]);
  for (idx_t m = 1; m < ct->nmodes; ++m) printf("->%" PRIu64 "", ct->dim_perm[m]);
  printf(")\n");
  printf("ntiles: %" PRIu64 " tile dims: %" PRIu64 "", ct->ntiles, ct->tile_dims[0]);
  for (idx_t m = 1; m < ct->nmodes; ++m) printf("x%" PRIu64 "", ct->tile_dims[m]);
  idx_t empty = 0;
  for (idx_t t = 0; t < ct->ntiles; ++t)
    if (ct->pt[t].vals == nullptr) ++empty;
  printf("  empty: %" PRIu64 " (%0.1f%%)\n", empty, 100. * (double)empty / (double)ct->ntiles);
}

void stats_csf_adaptive(splatt_csf const *const ct, idx_t const n_csf) {
  for (idx_t g = 0; g < n_csf; ++g) {
    printf("CSF-%" PRIu64 "\n", g);
    stats_one(ct + g);
  }
}

void stats_rcsf_adaptive(rcsf_seq_adaptive const *const seq_rcsfs, idx_t const n_rcsf) {
  for (idx_t g = 0; g < n_rcsf; ++g) {
    printf("vCSF Seq %" PRIu64 "\n", g);
    for (idx_t i = 0; i < seq_rcsfs[g].n_imten; ++i) {
      printf("   vCSF[%" PRIu64 "]:\n", i);
      stats_one(seq_rcsfs[g].rcsfs + i);
    }
  }
}

void iprint_array(idx_t const *const array, idx_t const len, char const *const name) {
  printf("%s: \n", name);
  for (idx_t i = 0; i < len; ++i) printf(" %" PRIu64, array[i]);
  printf("\n");
  fflush(stdout);
}

void print_group_properties(group_properties *const grp_prop, idx_t const size, idx_t const nmodes,
                            char *const name) {
  printf("====== %s =======\n", name);
  printf("[memo_mode, begin_imten, n_imten, o_opt]\n");
  for (idx_t i = 0; i < size; ++i) {
    printf("%" PRIu64 ", %" PRIu64 ", %" PRIu64 ", \n", grp_prop[i].memo_mode,
           grp_prop[i].begin_imten, grp_prop[i].n_imten);
    iprint_array(grp_prop[i].o_opt, nmodes, "o_opt");
  }
  printf("\n");
  fflush(stdout);
}

int adatm_rcsf_pull(rcsf_seq_adaptive *rs_seq, idx_t n_rcsf) {
  return guarded([&] {
    std::shared_ptr<CsfHandle> h;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      auto it = g_rcsf.find(rs_seq);
      if (it == g_rcsf.end()) throw BadInput("memo trees were not built by this library");
      h = it->second;
    }
    if (h->engines.empty()) throw BadInput("no engine");
    for (idx_t j = 0; j < n_rcsf; ++j) {
      const splatt_csf &r0 = rs_seq[j].rcsfs[0];
      const uint64_t R = r0.dims[r0.nmodes - 1];
      Engine &e = h->engine(R);
      int g = -1;  // the j-th memoizing tree
      for (int tt = 0, k = 0; tt < e.plan().n_csf; ++tt) {
        if (e.plan().tree(tt).n_imten == 0) continue;
        if ((idx_t)k == j) {
          g = tt;
          break;
        }
        ++k;
      }
      if (g < 0) throw BadInput("memo sequence index out of range");
      for (idx_t d = 0; d < rs_seq[j].n_imten; ++d) {
        const int rc = adatm_engine_memo_raw(&e, g, (int)d, rs_seq[j].rcsfs[d].pt->vals);
        if (rc != SPLATT_SUCCESS) throw BadInput(g_last_error);
      }
    }
  });
}

int adatm_csf_tree_count(splatt_csf const *tensors, int *n) {
  return guarded([&] { *n = find_csf(tensors)->n_csf; });
}

void adatm_free_groups(group_properties *grp_prop, idx_t n_grp) {
  if (!grp_prop) return;
  for (idx_t g = 0; g < n_grp; ++g) free(grp_prop[g].o_opt);
  free(grp_prop);
}

// ---------------------------------------------------------------------------
// device-resident interface
// ---------------------------------------------------------------------------
int adatm_tensor_from_coo(int nmodes, uint64_t nnz, const uint64_t *dims,
                          const uint64_t *const *inds, const double *vals, int clean,
                          adatm_tensor **out) {
  return guarded([&] {
    auto t = std::make_unique<adatm_tensor>();
    auto raw = upload_coo(nmodes, nnz, dims, inds, vals, t->stream.s);
    if (clean) {
      t->coo = std::make_shared<DevCoo>();
      coo_clean(*raw, *t->coo, t->stream.s);
    } else {
      t->coo = raw;
    }
    *out = t.release();
  });
}

int adatm_tensor_generate(int nmodes, const uint64_t *dims, uint64_t nnz, const double *alpha,
                          int value_kind, double mu, double sigma, uint64_t seed,
                          adatm_tensor **out) {
  return guarded([&] {
    auto t = std::make_unique<adatm_tensor>();
    DevCoo raw;
    coo_generate(raw, nmodes, dims, nnz, alpha, value_kind, mu, sigma, seed, t->stream.s);
    t->coo = std::make_shared<DevCoo>();
    coo_clean(raw, *t->coo, t->stream.s);
    *out = t.release();
  });
}

int adatm_tensor_info(const adatm_tensor *t, int *nmodes, uint64_t *nnz, uint64_t *dims) {
  return guarded([&] {
    if (nmodes) *nmodes = t->coo->nmodes;
    if (nnz) *nnz = t->coo->nnz;
    if (dims)
      for (int m = 0; m < t->coo->nmodes; ++m) dims[m] = t->coo->dims[m];
  });
}

int adatm_tensor_download(const adatm_tensor *t, uint64_t *inds, double *vals) {
  return guarded([&] {
    const DevCoo &c = *t->coo;
    std::vector<uint32_t> tmp(c.nnz);
    for (int m = 0; m < c.nmodes; ++m) {
      if (c.nnz == 0) continue;
      ADATM_CUDA(cudaMemcpyAsync(tmp.data(), c.idx[m].get(), c.nnz * 4, cudaMemcpyDeviceToHost,
                                 t->stream.s));
      ADATM_CUDA(cudaStreamSynchronize(t->stream.s));
      for (uint64_t n = 0; n < c.nnz; ++n) inds[(uint64_t)m * c.nnz + n] = tmp[n];
    }
    if (c.nnz)
      ADATM_CUDA(cudaMemcpyAsync(vals, c.vals.get(), c.nnz * sizeof(double),
                                 cudaMemcpyDeviceToHost, t->stream.s));
    ADATM_CUDA(cudaStreamSynchronize(t->stream.s));
  });
}

void adatm_tensor_free(adatm_tensor *t) { delete t; }

int adatm_tensor_count_nfibs(const adatm_tensor *t, const uint64_t *perm, uint64_t *nfibs) {
  return guarded([&] { csf_count(*t->coo, perm, nfibs, t->stream.s); });
}

int adatm_plan_analytic(const adatm_tensor *t, uint64_t rank, int strategy, adatm_plan *out,
                        adatm_candidate *cands, int max_cands, int *ncands, int *chosen) {
  return guarded([&] {
    std::vector<Candidate> all;
    Plan p = plan_analytic(*t->coo, rank, strategy, &all, t->stream.s);
    plan_to_c(p, out);
    if (ncands) *ncands = (int)all.size();
    if (chosen) *chosen = choose_candidate(all, strategy, 90e9);
    for (int i = 0; cands && i < (int)all.size() && i < max_cands; ++i) {
      Plan q = all[i].plan;
      decide_use_csfs(q);
      plan_to_c(q, &cands[i].plan);
      cands[i].pspace = all[i].pspace;
      cands[i].pops = all[i].pops;
    }
  });
}

int adatm_plan_splatt(const adatm_tensor *t, int csf_alloc, adatm_plan *out) {
  return guarded([&] {
    if (csf_alloc < SPLATT_CSF_ONEMODE || csf_alloc > SPLATT_CSF_ALLMODE)
      throw BadInput("csf_alloc must be ONEMODE, TWOMODE or ALLMODE");
    plan_to_c(plan_splatt(t->coo->nmodes, t->coo->dims, csf_alloc), out);
  });
}

int adatm_engine_create(const adatm_tensor *t, uint64_t rank, const adatm_plan *plan,
                        int factor_bf16, uint32_t chunk_leaf, uint32_t chunk_rows,
                        adatm_engine **out) {
  return guarded([&] {
    Plan p = plan_from_c(plan);
    if (p.nmodes != t->coo->nmodes) throw BadInput("plan order differs from the tensor's");
    check_plan(p);
    EngineOptions o;
    o.factor_type = factor_bf16 ? FactorType::BF16 : FactorType::F32;
    if (chunk_leaf) o.chunk_leaf = chunk_leaf;
    if (chunk_rows) o.chunk_rows = chunk_rows;
    auto e = std::make_unique<adatm_engine>();
    e->eng = std::make_unique<Engine>(t->coo, std::vector<std::shared_ptr<DevCsf>>{}, rank, p, o,
                                      e->stream.s);
    *out = e.release();
  });
}

void adatm_engine_free(adatm_engine *e) { delete e; }

int adatm_engine_csf_count(const adatm_engine *e, int *n_csf) {
  return guarded([&] { *n_csf = e->eng->n_csf(); });
}

int adatm_engine_csf_shape(const adatm_engine *e, int g, uint64_t *nfibs, uint64_t *dim_perm) {
  return guarded([&] {
    if (g < 0 || g >= e->eng->n_csf()) throw BadInput("tree index out of range");
    const DevCsf &c = e->eng->csf(g);
    for (int l = 0; l < c.nmodes; ++l) {
      nfibs[l] = c.nfibs[l];
      dim_perm[l] = c.dim_perm[l];
    }
  });
}

int adatm_engine_csf_arrays(const adatm_engine *e, int g, uint64_t *const *fptr,
                            uint64_t *const *fids, double *vals) {
  return guarded([&] {
    if (g < 0 || g >= e->eng->n_csf()) throw BadInput("tree index out of range");
    const DevCsf &c = e->eng->csf(g);
    HostCsfArrays a;
    csf_download(c, a, e->stream.s);
    for (int l = 0; l < c.nmodes; ++l) {
      if (l < c.nmodes - 1 && fptr && fptr[l]) memcpy(fptr[l], a.fptr[l].data(), a.fptr[l].size() * 8);
      if (fids && fids[l]) memcpy(fids[l], a.fids[l].data(), a.fids[l].size() * 8);
    }
    if (vals) memcpy(vals, a.vals.data(), a.vals.size() * 8);
  });
}

int adatm_engine_memory(const adatm_engine *e, uint64_t *csf_bytes, uint64_t *memo_bytes) {
  return guarded([&] {
    if (csf_bytes) *csf_bytes = e->eng->csf_bytes();
    if (memo_bytes) *memo_bytes = e->eng->memo_bytes();
  });
}

int adatm_engine_init_factors(adatm_engine *e, uint64_t seed) {
  return guarded([&] { e->eng->init_factors(seed); });
}

int adatm_engine_set_factors(adatm_engine *e, const double *const *mats) {
  return guarded([&] { e->eng->set_factors(mats); });
}

int adatm_engine_get_factors(adatm_engine *e, double *const *mats, double *lambda) {
  return guarded([&] {
    if (mats) e->eng->get_factors(mats);
    if (lambda) e->eng->get_lambda(lambda);
  });
}


int adatm_engine_mttkrp(adatm_engine *e, uint64_t mode, double *out) {
  return guarded([&] {
    Engine &g = *e->eng;
    if (mode >= (uint64_t)g.nmodes()) throw BadInput("mode out of range");
    g.mttkrp((int)mode, g.mttkrp_buffer());
    pull_rows(g, g.mttkrp_buffer(), g.dims()[mode], out);
  });
}

int adatm_engine_mttkrp_direct(adatm_engine *e, uint64_t mode, double *out) {
  return guarded([&] {
    Engine &g = *e->eng;
    if (mode >= (uint64_t)g.nmodes()) throw BadInput("mode out of range");
    g.mttkrp_direct((int)mode, g.mttkrp_buffer());
    pull_rows(g, g.mttkrp_buffer(), g.dims()[mode], out);
  });
}

int adatm_engine_memo(adatm_engine *e, int g, int deg, double *out) {
  return adatm_engine_memo_raw(e->eng.get(), g, deg, out);
}

int adatm_engine_als(adatm_engine *e, uint64_t niters, double tol, int use_graph, double *fit,
                     uint64_t *iters, double *trace) {
  return guarded([&] {
    Engine &g = *e->eng;
    g.als_begin();
    if (use_graph) g.capture_graph();
    double f = 0, old = 0;
    uint64_t it = 0;
    for (it = 0; it < niters; ++it) {
      g.sweep();
      if (tol > 0 || it + 1 == niters) {
        f = g.fit_host();
        if (it > 0 && std::fabs(f - old) < tol) {
          ++it;
          break;
        }
        old = f;
      }
    }
    f = g.fit_host();
    if (fit) *fit = f;
    if (iters) *iters = it;
    if (trace) g.fit_trace(trace, (int)it);
  });
}

int adatm_engine_als_begin(adatm_engine *e, int use_graph) {
  return guarded([&] {
    e->eng->als_begin();
    if (use_graph) e->eng->capture_graph();
  });
}

int adatm_engine_time_sweeps(adatm_engine *e, int count, float *ms) {
  return guarded([&] {
    Engine &g = *e->eng;
    cudaEvent_t a, b;
    ADATM_CUDA(cudaEventCreate(&a));
    ADATM_CUDA(cudaEventCreate(&b));
    ADATM_CUDA(cudaStreamSynchronize(g.stream()));
    ADATM_CUDA(cudaEventRecord(a, g.stream()));
    for (int i = 0; i < count; ++i) g.sweep();
    ADATM_CUDA(cudaEventRecord(b, g.stream()));
    ADATM_CUDA(cudaEventSynchronize(b));
    ADATM_CUDA(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

int adatm_engine_time_mttkrp(adatm_engine *e, uint64_t mode, int count, float *ms) {
  return guarded([&] {
    Engine &g = *e->eng;
    if (mode >= (uint64_t)g.nmodes()) throw BadInput("mode out of range");
    cudaEvent_t a, b;
    ADATM_CUDA(cudaEventCreate(&a));
    ADATM_CUDA(cudaEventCreate(&b));
    ADATM_CUDA(cudaStreamSynchronize(g.stream()));
    ADATM_CUDA(cudaEventRecord(a, g.stream()));
    for (int i = 0; i < count; ++i) g.mttkrp_as((int)mode, g.mttkrp_buffer(), g.sweep_type((int)mode));
    ADATM_CUDA(cudaEventRecord(b, g.stream()));
    ADATM_CUDA(cudaEventSynchronize(b));
    ADATM_CUDA(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

int adatm_engine_fit(adatm_engine *e, double *fit) {
  return guarded([&] { *fit = e->eng->fit_host(); });
}

int adatm_engine_mttkrp_into(adatm_engine *e, uint64_t mode, double *dev_out) {
  return guarded([&] {
    if (!e || !dev_out) throw BadInput("adatm_engine_mttkrp_into: null argument");
    if (mode >= (uint64_t)e->eng->nmodes()) throw BadInput("mode out of range");
    e->eng->mttkrp_into((int)mode, dev_out);
  });
}

int adatm_engine_update_from(adatm_engine *e, uint64_t mode, const double *dev_M) {
  return guarded([&] {
    if (!e || !dev_M) throw BadInput("adatm_engine_update_from: null argument");
    e->eng->update_from((int)mode, dev_M);
  });
}

int adatm_engine_fit_step(adatm_engine *e, double *fit) {
  return guarded([&] { *fit = e->eng->fit_step(); });
}

int adatm_engine_ttnorm(adatm_engine *e, double *local) {
  return guarded([&] { *local = e->eng->ttnorm_local(); });
}

int adatm_engine_set_ttnorm(adatm_engine *e, double global) {
  return guarded([&] { e->eng->set_ttnorm(global); });
}

int adatm_engine_mttkrp_bytes(adatm_engine *e, uint64_t mode, double *bytes) {
  return guarded([&] {
    if (mode >= (uint64_t)e->eng->nmodes()) throw BadInput("mode out of range");
    *bytes = e->eng->mttkrp_bytes((int)mode);
  });
}

int adatm_engine_hot_rows(adatm_engine *e, uint64_t mode, int *nhot) {
  return guarded([&] {
    if (!e || !nhot) throw BadInput("adatm_engine_hot_rows: null argument");
    if (mode >= (uint64_t)e->eng->nmodes()) throw BadInput("mode out of range");
    *nhot = e->eng->walk((int)mode).nhot;
  });
}

int adatm_engine_autotune(adatm_engine *e, const uint32_t *chunk_leaf, const uint32_t *chunk_rows,
                          int n, int sweeps, int *best) {
  return guarded([&] {
    if (n < 1 || !chunk_leaf || !chunk_rows) throw BadInput("adatm_engine_autotune: no options");
    std::vector<std::pair<uint32_t, uint32_t>> opts;
    for (int i = 0; i < n; ++i) opts.emplace_back(chunk_leaf[i], chunk_rows[i]);
    const int b = e->eng->autotune(opts, sweeps);
    e->graph = false;
    if (best) *best = b;
  });
}

int adatm_engine_set_resident_grid(adatm_engine *e, int on) {
  return guarded([&] {
    if (!e) throw BadInput("adatm_engine_set_resident_grid: null engine");
    e->eng->set_resident_grid(on != 0);
    e->graph = false;
  });
}

int adatm_engine_set_walkers(adatm_engine *e, int walkers) {
  return guarded([&] {
    if (!e) throw BadInput("adatm_engine_set_walkers: null engine");
    e->eng->set_walkers(walkers);
    e->graph = false;
  });
}

int adatm_engine_set_fold(adatm_engine *e, int fold) {
  return guarded([&] {
    if (!e) throw BadInput("adatm_engine_set_fold: null engine");
    e->eng->set_fold(fold);
    e->graph = false;
  });
}

int adatm_engine_set_deterministic(adatm_engine *e, int on) {
  return guarded([&] {
    if (!e) throw BadInput("adatm_engine_set_deterministic: null engine");
    e->eng->set_deterministic(on != 0);
    e->graph = false;
  });
}

int adatm_batch_create(adatm_engine *const *engines, int n, adatm_batch **out) {
  return guarded([&] {
    if (n < 1 || !engines || !out) throw BadInput("adatm_batch_create: no engines");
    std::vector<Engine *> es;
    for (int i = 0; i < n; ++i) {
      if (!engines[i]) throw BadInput("adatm_batch_create: null engine");
      es.push_back(engines[i]->eng.get());
    }
    auto b = std::make_unique<adatm_batch>();
    b->batch = std::make_unique<BatchSweep>(es, b->stream.s);
    *out = b.release();
  });
}

int adatm_batch_begin(adatm_batch *b) {
  return guarded([&] { b->batch->begin(); });
}

int adatm_batch_time_sweeps(adatm_batch *b, int count, float *ms) {
  return guarded([&] { *ms = b->batch->time_sweeps(count); });
}

int adatm_batch_kernels(const adatm_batch *b, int *per_sweep) {
  return guarded([&] { *per_sweep = b->batch->kernels_per_sweep(); });
}

void adatm_batch_free(adatm_batch *b) { delete b; }

int adatm_plan_features(const adatm_tensor *t, uint64_t rank, float *features, double *bytes,
                        adatm_candidate *cands, int max_cands, int *ncands) {
  return guarded([&] {
    if (!t || rank < 1) throw BadInput("adatm_plan_features: no tensor or rank 0");
    std::vector<Candidate> all = candidate_configs(t->coo->nmodes, t->coo->dims);
    predict_candidates(*t->coo, rank, all, t->stream.s);
    std::vector<float> f;
    std::vector<double> b;
    plan_features(*t->coo, rank, all, f, b, t->stream.s);
    if (ncands) *ncands = (int)all.size();
    for (int i = 0; i < (int)all.size() && i < max_cands; ++i) {
      if (features) memcpy(features + (size_t)i * kPlanFeatures, &f[(size_t)i * kPlanFeatures],
                           kPlanFeatures * sizeof(float));
      if (bytes) bytes[i] = b[i];
      if (cands) {
        Plan q = all[i].plan;
        decide_use_csfs(q);
        plan_to_c(q, &cands[i].plan);
        cands[i].pspace = all[i].pspace;
        cands[i].pops = all[i].pops;
      }
    }
  });
}

int adatm_mlp_create(int nwidths, const int *widths, uint64_t seed, adatm_mlp **out) {
  return guarded([&] {
    if (nwidths < 2 || !widths || !out) throw BadInput("adatm_mlp_create: bad widths");
    auto m = std::make_unique<adatm_mlp>();
    m->net = std::make_unique<Mlp>(std::vector<int>(widths, widths + nwidths), seed, m->stream.s);
    *out = m.release();
  });
}

void adatm_mlp_free(adatm_mlp *m) { delete m; }

int adatm_mlp_nparams(const adatm_mlp *m, uint64_t *n) {
  return guarded([&] { *n = m->net->nparams(); });
}

int adatm_mlp_set_params(adatm_mlp *m, const float *params) {
  return guarded([&] { m->net->set_params(params); });
}

int adatm_mlp_get_params(const adatm_mlp *m, float *params) {
  return guarded([&] { m->net->get_params(params); });
}

int adatm_mlp_forward(adatm_mlp *m, const float *X, uint64_t rows, float *Y) {
  return guarded([&] {
    if (rows > (1u << 30)) throw BadInput("adatm_mlp_forward: too many rows");
    m->net->forward(X, (int)rows, Y);
  });
}

int adatm_mlp_gradient(adatm_mlp *m, const float *X, const float *T, uint64_t rows, float *grad,
                       double *loss) {
  return guarded([&] {
    if (rows == 0 || rows > (1u << 30)) throw BadInput("adatm_mlp_gradient: bad row count");
    const double l = m->net->gradient(X, T, (int)rows, grad);
    if (loss) *loss = l;
  });
}

int adatm_mlp_train(adatm_mlp *m, const float *X, const float *T, uint64_t rows, int epochs,
                    int batch, float lr, uint64_t seed, double *loss) {
  return guarded([&] {
    const double l = m->net->train(X, T, rows, epochs, batch, lr, seed);
    if (loss) *loss = l;
  });
}

int adatm_plan_learned(const adatm_tensor *t, uint64_t rank, adatm_mlp *m, const float *feat_mean,
                       const float *feat_std, adatm_plan *out, int *chosen, int *used_model) {
  return guarded([&] {
    std::vector<Candidate> all = candidate_configs(t->coo->nmodes, t->coo->dims);
    predict_candidates(*t->coo, rank, all, t->stream.s);
    int pick = -1;
    if (m && feat_mean && feat_std && m->net->widths()[0] == kPlanFeatures) {
      std::vector<float> f;
      std::vector<double> b;
      plan_features(*t->coo, rank, all, f, b, t->stream.s);
      for (size_t i = 0; i < f.size(); ++i) {
        const int k = (int)(i % kPlanFeatures);
        f[i] = (f[i] - feat_mean[k]) / (feat_std[k] > 0 ? feat_std[k] : 1.f);
      }
      std::vector<float> y(all.size());
      m->net->forward(f.data(), (int)all.size(), y.data());
      bool finite = true;
      for (float v : y) finite = finite && std::isfinite(v);
      if (finite)
        for (size_t c = 0; c < all.size(); ++c)
          if (b[c] < 90e9 && (pick < 0 || y[c] < y[pick])) pick = (int)c;
    }
    if (used_model) *used_model = pick >= 0 ? 1 : 0;
    if (pick < 0) pick = choose_candidate(all, 1, 90e9);
    if (pick < 0) throw NoMemory("no memoization plan fits the storage limit");
    Plan p = all[pick].plan;
    decide_use_csfs(p);
    plan_to_c(p, out);
    if (chosen) *chosen = pick;
  });
}

int adatm_gram(const float *A, uint64_t rows, int R, int ldr, double *G) {
  return guarded([&] {
    if (R < 1 || R > 128 || ldr < R || ldr % 4 != 0) throw BadInput("adatm_gram: bad R or ldr");
    if (((uintptr_t)A & 15) != 0) throw BadInput("adatm_gram: A must be 16-byte aligned");
    StreamOwner s;
    int dev = 0, sms = 148;
    ADATM_CUDA(cudaGetDevice(&dev));
    ADATM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    AlsWork w;
    w.init(1, R, 2 * sms, 1);
    w.ldr = ldr;
    gram(A, rows, R, ldr, G, w, s.s);
    ADATM_CUDA(cudaStreamSynchronize(s.s));
  });
}

int adatm_gram_noalloc(const float *A, uint64_t rows, int R, int ldr, double *G, void *stream) {
  return guarded([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    gram_noalloc(A, rows, R, ldr, G, s);
    ADATM_CUDA(cudaStreamSynchronize(s));
  });
}

int adatm_engine_launch_counts(adatm_engine *e, uint64_t mode, int *per_sweep, int *per_mttkrp) {
  return guarded([&] {
    if (per_sweep) *per_sweep = e->eng->kernels_per_sweep();
    if (per_mttkrp) *per_mttkrp = e->eng->kernels_per_mttkrp((int)mode);
  });
}

}  // extern "C"

namespace {
int adatm_engine_memo_raw(Engine *g, int grp, int deg, double *out) {
  // grp: tree index (the group index in TIME_EFFICIENT plans)
  return guarded([&] {
    const Plan &p = g->plan();
    if (grp < 0 || grp >= p.n_csf || deg < 0 || (uint64_t)deg >= p.tree(grp).n_imten)
      throw BadInput("memo tree out of range");
    const uint64_t lvl = p.tree(grp).begin_imten - 1 - deg;
    const uint64_t rows = g->csf(grp).nfibs[lvl];
    pull_rows(*g, g->memo_rows(grp, deg), rows, out);
  });
}
}  // namespace
