// Launch-shape autotuner with a persisted cache: tile size (elements per
// CTA), threads per CTA and, for VMS, the register budget (the tile kernel
// variant compiled for 3 or 4 resident 128-thread CTAs an SM, ...).
#include <unistd.h>

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fm_internal.hpp"

namespace fm {
int vms_default_ctas(int threads, bool mixed);
bool vms_variant_exists(int threads, bool mixed, int ctas);
}  // namespace fm

namespace {

std::string cache_key(fm_problem* const* probs, int n, int device) {
  cudaDeviceProp prop;
  std::string gpu = "unknown";
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) gpu = prop.name;
  for (auto& c : gpu)
    if (c == ' ') c = '_';
  int64_t E = 0;
  for (int i = 0; i < n; ++i) E += probs[i]->E;
  int lg = 0;
  while ((int64_t(1) << (lg + 1)) <= E) ++lg;
  std::ostringstream k;
  k << gpu << "/s" << probs[0]->params.solver << "/e" << probs[0]->etype << "/p" << probs[0]->params.precision << "/n"
    << (n > 1 ? 1 : 0) << "/E2^" << lg;
  return k.str();
}

bool cache_lookup(const char* path, const std::string& key, fm_tuning* t) {
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream l(line);
    std::string k;
    int te = 0, tn = 0, th = 0, ctas = 0;
    if (!(l >> k >> te >> tn >> th) || k != key) continue;
    l >> ctas;  // absent in lines written before the register budget was tuned
    memset(t, 0, sizeof(*t));
    t->tile_elems = te;
    t->tile_nodes = tn;
    t->threads = th;
    t->ctas_per_sm = ctas;
    return true;
  }
  return false;
}

void cache_store(const char* path, const std::string& key, const fm_tuning& t) {
  if (!path) return;
  std::vector<std::string> lines;
  {
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line))
      if (line.compare(0, key.size() + 1, key + " ") != 0 && !line.empty()) lines.push_back(line);
  }
  std::ostringstream l;
  l << key << " " << t.tile_elems << " " << t.tile_nodes << " " << t.threads << " " << t.ctas_per_sm;
  lines.push_back(l.str());
  // written whole to a file of this process and renamed over the cache, so
  // a reader (or another rank storing at the same time) sees an old or a new
  // complete file, never a partial one
  const std::string tmp = std::string(path) + ".tmp" + std::to_string((long long)getpid());
  {
    std::ofstream f(tmp, std::ios::trunc);
    for (auto& s : lines) f << s << "\n";
    if (!f.good()) {
      f.close();
      std::remove(tmp.c_str());
      return;
    }
  }
  if (std::rename(tmp.c_str(), path) != 0) std::remove(tmp.c_str());
}

}  // namespace

extern "C" int fm_autotune(fm_problem* const* probs, int32_t n, int32_t device, int32_t steps, const char* cache_path,
                           fm_tuning* best) {
  fm::NvtxRange nvtx_range("fm_autotune");
  if (!probs || n <= 0 || !best) return fm::fail(FM_ERR_INVALID, "null argument");
  for (int i = 0; i < n; ++i)
    if (!probs[i] || probs[i]->batch) return fm::fail(FM_ERR_INVALID, "problems must exist and not be in a batch");
  const std::string key = cache_key(probs, n, device);
  if (cache_lookup(cache_path, key, best)) return FM_OK;
  const bool hexa = probs[0]->etype == 8;
  const bool vms = probs[0]->params.solver == FM_SOLVER_VMS;
  struct Cand {
    int te, tn, th, ctas;
  };
  std::vector<Cand> cands;
  if (vms) {
    const bool mixed = probs[0]->params.precision == FM_MIXED;
    for (int th : {128, 256}) {
      const int c0 = fm::vms_default_ctas(th, mixed);
      for (int ctas : {c0, c0 + 1}) {
        if (!fm::vms_variant_exists(th, mixed, ctas)) continue;
        for (int te : {384, 512, 768, 1024}) cands.push_back({te, FM_MAX_TILE_NODES, th, ctas});
      }
    }
  } else if (hexa) {
    for (int th : {128, 256})
      for (int te : {128, 256, 384, 512}) cands.push_back({te, 2 * te + 256, th, 0});
  } else {
    for (int th : {128, 256})
      for (int te : {512, 1024, 2048}) cands.push_back({te, te / 2 + 128, th, 0});
  }
  double best_ms = 1e300;
  fm_tuning bt;
  memset(&bt, 0, sizeof(bt));
  if (steps <= 0) steps = 10;
  for (const Cand& c : cands) {
    fm_tuning t;
    memset(&t, 0, sizeof(t));
    t.tile_elems = c.te;
    t.tile_nodes = c.tn;
    t.threads = c.th;
    t.ctas_per_sm = c.ctas;
    fm_batch* b = nullptr;
    if (fm_batch_create(probs, n, &t, device, &b) != FM_OK) continue;
    double ms[2] = {0, 0};
    int64_t ln[2] = {0, 0};
    int r = fm_batch_step(b, 2, nullptr);
    if (!r) r = fm_batch_sync(b);
    if (!r) r = fm_batch_profile(b, steps, ms, ln);
    fm_batch_destroy(b);
    if (r) continue;
    const double per = (ms[0] + ms[1]) / (double)(ln[0] > 0 ? ln[0] : 1);
    if (per < best_ms) {
      best_ms = per;
      bt = t;
    }
  }
  for (int i = 0; i < n; ++i) probs[i]->steps_done = 0;
  if (best_ms >= 1e300) return fm::fail(FM_ERR_CUDA, "autotune: no candidate ran");
  *best = bt;
  cache_store(cache_path, key, bt);
  return FM_OK;
}
