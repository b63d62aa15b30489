// espp_api.cu - host runtime and C ABI (include/espp_b200.h) of the B200 MD step.
//
// One espp_system owns all particles of one box on the current CUDA device, in
// cell-sorted SoA arrays (two copies, swapped at each re-sort), plus the Verlet list,
// force buffers and the device scalars of the rebuild criterion.  The run loop follows
// VelocityVerlet::run (src/integrator/VelocityVerlet.cpp:63-169): start-of-run force
// with the Langevin heat-up factor, then per step integrate1 -> (re-sort + list build
// when the accumulated max displacement exceeds skin/2) -> forces -> aftCalcF ->
// integrate2.  integrate2 of step n and integrate1 of step n+1 run as one kernel.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/espp_b200.h"
#include "espp_internal.h"
#include "espp_tab.h"
#include "espp_mlp.h"

using namespace espp;

namespace {

thread_local std::string g_err;

struct Fail {
  int code;
  std::string msg;
};

[[noreturn]] void raise(int code, const std::string& msg) { throw Fail{code, msg}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    raise(ESPP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* dalloc(size_t count) {
  void* p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(&p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    raise(ESPP_ENOMEM, std::string("device allocation of ") +
                           std::to_string(count * sizeof(T)) + " bytes failed");
  }
  return (T*)p;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

}  // namespace

struct espp_system {
  // configuration
  double L[3];
  double skin;
  int nc[3];
  int hci = 1;  // halfCellInt
  int precision;
  uint64_t seed;
  int device = 0;
  cudaStream_t st = nullptr;

  // particles on the device
  int n = 0, cap = 0;
  ParticleArrays A{}, B{};
  int4* posq = nullptr;
  float4* xrel = nullptr;
  int32_t* pcell = nullptr;
  int32_t* cellStart = nullptr;
  int32_t* nl = nullptr;
  int32_t* nn = nullptr;
  int32_t* nnZero = nullptr;  // all-zero counts (no pair interaction)
  int K = 0;
  long long* ffix = nullptr;
  double* f64 = nullptr;
  double* ftot = nullptr;
  RebuildScratch scr{};
  bool binned = false;
  bool listValid = false;
  bool xrelFresh = false;  // xrel written by the last gather from the current positions

  // staging for by-id state transfers
  int stageCap = 0;
  int64_t* stIds = nullptr;
  double* stPos = nullptr;
  double* stVel = nullptr;
  double* stF = nullptr;
  int32_t* stImg = nullptr;

  // device-event timing of the run loop
  bool profiling = false;
  std::vector<cudaEvent_t> evPool;
  size_t evUsed = 0;
  std::vector<std::pair<int, size_t>> evPhase;  // (phase, index of start event)
  double phaseMs[8] = {0};                      // force, integrate, re-sort, decide, list
  long long phaseLaunches[8] = {0};
  cudaEvent_t runBeg = nullptr, runLoop = nullptr, runEnd = nullptr;
  double lastRunMs = 0.0, lastLoopMs = 0.0;

  // id-indexed structures
  int64_t idMin = 0;
  int idSpan = 0;
  int32_t* id2idx = nullptr;
  int32_t* bondStart = nullptr;
  int64_t* bondPartner = nullptr;
  uint8_t* langExcl = nullptr;
  uint8_t* halo = nullptr;  // idSpan, built when haloIds is not empty
  int32_t* exclStart = nullptr;
  int64_t* exclIds = nullptr;
  bool idDirty = true;

  // device scalars
  unsigned* err = nullptr;
  DevCounters* ctr = nullptr;     // device
  DevCounters* hctr = nullptr;    // pinned host mirror
  ParticleArrays* d_pa = nullptr; // device: [0] current, [1] re-sort target
  bool paHostValid = true;        // host A/B mirror what d_pa holds
  double* obs = nullptr;
  double* partials = nullptr;
  int partialsCap = 0;

  // captured step loop (WHILE { decide; IF(re-sort) {...}; force; integrate })
  bool useGraph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  std::string graphKey;
  // pre-run snapshot to recover from a Verlet-list overflow inside the graph
  ParticleArrays snap{};
  int snapCap = 0;

  // brick path of the Verlet list and pair kernels (BrickView)
  bool brickAllowed = false;  // ESPP_B200_BRICK=1 selects the brick form
  bool brickBuild = false;    // the global-form list is built by brick windows
                              // (ESPP_B200_BRICK_BUILD=1) instead of the per-cell lanes
  bool brickBuildUsed = false;  // the current global-form list came from the brick build
  bool brickOn = false;       // the current list is in the brick form
  int brickB[3] = {0, 0, 0};  // brick extent in cells (0: chosen from the density)
  int brickWmax = 0;          // window slots (sentinel included)
  uint16_t* bnl = nullptr;    // bKb * cap entries
  int bKb = 0;
  double* bpartials = nullptr;  // one row of 7 per brick (observables, digest)
  int bpartialsCap = 0;

  // Verlet list
  bool has_vl = false;
  double vl_cut = 0.0;
  std::vector<std::pair<int64_t, int64_t>> vlExcl;
  int64_t builds = 0;

  // potentials
  LJTable lj{};
  LJPair* d_lj = nullptr;
  LJPairF* d_ljf = nullptr;
  bool lj_any = false;
  FENEParams fene{};
  std::vector<std::pair<int64_t, int64_t>> bonds;
  // FixedTripleList + Cosine
  std::vector<std::array<int64_t, 3>> triples;
  CosineParams cosine{};
  int64_t* d_triples = nullptr;
  int32_t* tripStart = nullptr;
  int32_t* tripEntry = nullptr;
  double* tripF = nullptr;
  // interaction::Tabulated: specifications by slot (type pair key t1*kMaxTypes+t2 with
  // t1 <= t2, or kTabBondKey for the fixed pair list), built into one coefficient array
  struct TabSpec {
    int itype;
    std::vector<double> r, e, f;
    double rc, shift;
  };
  std::map<int, TabSpec> tabSpecs;
  TabDesc* d_tabs = nullptr;
  double* d_tabCoef = nullptr;
  int32_t* d_tabPair = nullptr;
  int tabNT = 0;
  int tabBond = -1;
  int tabAngle = -1;
  // learned CG potential (not owned) and its per-particle scratch
  espp_mlp* mlp = nullptr;
  int mlpCap = 0;
  float* mlpG = nullptr;
  float* mlpD = nullptr;
  float* mlpE = nullptr;
  float* mlpF = nullptr;    // force-matching: model force, error adjoint, tangent
  float* mlpErr = nullptr;
  float* mlpTan = nullptr;
  float* mlpPart = nullptr;
  double* mlpFref = nullptr;
  // sums of total forces by particle id (espp_force_acc)
  double* facc = nullptr;
  int faccSpan = 0;

  // integrator
  double dt = 0.005;
  int64_t step = 0;
  int64_t nResorts = 0;
  bool resortFlag = true;
  bool lang_on = false;
  double gamma = 0.0, temperature = 0.0;
  std::vector<int64_t> langExclIds;
  // spatial decomposition: ids of the halo copies of other domains' particles, and the
  // step-loop state of a run driven step by step by the decomposition's host loop
  std::vector<int64_t> haloIds;
  bool ddRun = false;
  int64_t ddSteps = 0, ddDone = 0;
  double ddT0 = 0.0, ddTResort = 0.0;
  IntegrateArgs ddArgs{};
  int capMode = ESPP_CAP_OFF;
  double cap3[3] = {0, 0, 0};
  int tpp = 4;
  double timers[10] = {0};

  // host id list (all particle ids, for the id map) and the largest type present
  std::vector<int64_t> allIds;
  int maxType = 0;

  BrickView brick_view() const {
    BrickView b{};
    b.on = brickOn ? 1 : 0;
    b.nbricks = 1;
    for (int k = 0; k < 3; ++k) {
      b.b[k] = brickB[k] > 0 ? brickB[k] : 1;
      b.nb[k] = (nc[k] + b.b[k] - 1) / b.b[k];
      b.nbricks *= b.nb[k];
    }
    b.wmax = brickWmax;
    b.nl = bnl;
    b.Kb = bKb;
    return b;
  }

  DevView view() const {
    DevView d{};
    d.pa = d_pa;
    d.n = n;
    d.cap = cap;
    for (int k = 0; k < 3; ++k) {
      d.L[k] = L[k];
      d.invL[k] = 1.0 / L[k];
      d.halfL[k] = 0.5 * L[k];
      d.cellSize[k] = (L[k] - 0.0) / double(nc[k]);
      d.invCellSize[k] = 1.0 / d.cellSize[k];
      d.nc[k] = nc[k];
      d.fixScale[k] = kFix / L[k];
      d.fixUnit[k] = (float)(L[k] / kFix);
    }
    d.ncells = nc[0] * nc[1] * nc[2];
    d.hci = hci;
    d.posq = posq;
    d.xrel = xrel;
    d.pcell = pcell;
    d.cellStart = cellStart;
    d.nl = nl;
    d.nn = nn;
    d.K = K;
    d.ffix = ffix;
    d.f64 = f64;
    d.ftot = ftot;
    d.idMin = idMin;
    d.idSpan = idSpan;
    d.id2idx = id2idx;
    d.bondStart = bondStart;
    d.bondPartner = bondPartner;
    d.langExcl = langExcl;
    d.halo = halo;
    d.exclStart = exclStart;
    d.exclIds = exclIds;
    d.lj = d_lj;
    d.ljf = d_ljf;
    d.ntypes = lj.ntypes;
    d.ljSingle = lj.single;
    int capped = 0;
    for (int k = 0; k < kMaxTypes * kMaxTypes; ++k)
      if (lj.p[k].set && lj.p[k].caprad > 0) capped = 1;
    d.ljCapped = capped;
    d.tabs = d_tabs;
    d.tabCoef = d_tabCoef;
    d.tabPair = d_tabPair;
    d.tabNT = tabNT;
    d.tabBond = tabBond;
    d.tabAngle = tabAngle;
    d.mlp = mlp_view(mlp);
    d.mlp.G = mlpG;
    d.mlp.D = mlpD;
    d.mlp.E = mlpE;
    d.mlp.on = (mlp && has_vl) ? 1 : 0;
    d.triples = d_triples;
    d.ntriples = (int)triples.size();
    d.tripStart = tripStart;
    d.tripEntry = tripEntry;
    d.tripF = tripF;
    d.cosine = cosine;
    d.brick = brick_view();
    d.err = err;
    d.ctr = ctr;
    return d;
  }
};

namespace {

void free_particles(ParticleArrays& a) {
  dfree(a.x);
  dfree(a.v);
  dfree(a.id);
  dfree(a.type);
  dfree(a.mass);
  dfree(a.img);
}

void alloc_particles(ParticleArrays& a, int cap) {
  a.x = dalloc<double>(3 * (size_t)cap);
  a.v = dalloc<double>(3 * (size_t)cap);
  a.id = dalloc<int64_t>(cap);
  a.type = dalloc<int32_t>(cap);
  a.mass = dalloc<double>(cap);
  a.img = dalloc<int32_t>(3 * (size_t)cap);
}

void sync(espp_system* s) { cuda_check(cudaStreamSynchronize(s->st), "stream synchronize"); }

// Host view of which physical buffers are current (the re-sort swaps them on the device).
void sync_pa(espp_system* s) {
  if (s->paHostValid) return;
  ParticleArrays h[2];
  cuda_check(cudaMemcpyAsync(h, s->d_pa, sizeof(h), cudaMemcpyDeviceToHost, s->st), "arrays");
  sync(s);
  s->A = h[0];
  s->B = h[1];
  s->paHostValid = true;
}

void push_pa(espp_system* s) {
  ParticleArrays h[2] = {s->A, s->B};
  cuda_check(cudaMemcpyAsync(s->d_pa, h, sizeof(h), cudaMemcpyHostToDevice, s->st), "arrays");
  sync(s);
  s->paHostValid = true;
}

// Host copy of every particle in storage order.
struct HostParticles {
  std::vector<int64_t> id;
  std::vector<int32_t> type, img;
  std::vector<double> mass, x, v, f;  // interleaved 3-vectors
};

template <class T>
void copy_soa_down(espp_system* s, std::vector<T>& out, const T* dsrc, int comps) {
  std::vector<T> tmp((size_t)comps * s->cap);
  if (s->cap)
    cuda_check(cudaMemcpy(tmp.data(), dsrc, sizeof(T) * tmp.size(), cudaMemcpyDeviceToHost),
               "download");
  out.resize((size_t)comps * s->n);
  for (int i = 0; i < s->n; ++i)
    for (int c = 0; c < comps; ++c) out[(size_t)comps * i + c] = tmp[(size_t)c * s->cap + i];
}

HostParticles download(espp_system* s, bool withForce) {
  sync_pa(s);
  HostParticles h;
  copy_soa_down(s, h.id, s->A.id, 1);
  copy_soa_down(s, h.type, s->A.type, 1);
  copy_soa_down(s, h.mass, s->A.mass, 1);
  copy_soa_down(s, h.x, s->A.x, 3);
  copy_soa_down(s, h.v, s->A.v, 3);
  copy_soa_down(s, h.img, s->A.img, 3);
  if (withForce) copy_soa_down(s, h.f, s->ftot, 3);
  return h;
}

template <class T>
void copy_soa_up(espp_system* s, T* ddst, const std::vector<T>& in, int comps) {
  std::vector<T> tmp((size_t)comps * s->cap, T(0));
  for (int i = 0; i < s->n; ++i)
    for (int c = 0; c < comps; ++c) tmp[(size_t)c * s->cap + i] = in[(size_t)comps * i + c];
  cuda_check(cudaMemcpy(ddst, tmp.data(), sizeof(T) * tmp.size(), cudaMemcpyHostToDevice),
             "upload");
}

void free_buffers(espp_system* s) {
  free_particles(s->A);
  free_particles(s->B);
  dfree(s->posq);
  dfree(s->xrel);
  dfree(s->pcell);
  dfree(s->nl);
  dfree(s->nn);
  dfree(s->nnZero);
  dfree(s->ffix);
  dfree(s->f64);
  dfree(s->ftot);
  dfree(s->scr.cellOf);
  dfree(s->scr.slot);
  dfree(s->scr.perm);
}

// Reallocates the per-particle buffers for cap >= n and uploads h.
void ensure_mlp_scratch(espp_system* s);

void upload(espp_system* s, const HostParticles& h) {
  int n = (int)h.id.size();
  sync_pa(s);
  if (n > s->cap) {
    free_buffers(s);
    int cap = std::max(n, 32);
    cap = (cap + 31) / 32 * 32;
    s->cap = cap;
    alloc_particles(s->A, cap);
    alloc_particles(s->B, cap);
    s->posq = dalloc<int4>(cap);
    s->xrel = dalloc<float4>(cap);
    s->pcell = dalloc<int32_t>(cap);
    s->nn = dalloc<int32_t>(cap);
    s->nnZero = dalloc<int32_t>(cap);
    cuda_check(cudaMemset(s->nnZero, 0, sizeof(int32_t) * cap), "memset");
    s->ffix = dalloc<long long>(3 * (size_t)cap);
    s->f64 = dalloc<double>(3 * (size_t)cap);
    s->ftot = dalloc<double>(3 * (size_t)cap);
    s->scr.cellOf = dalloc<int32_t>(cap);
    s->scr.slot = dalloc<int32_t>(cap);
    s->scr.perm = dalloc<int32_t>(cap);
    cuda_check(cudaMemset(s->nn, 0, sizeof(int32_t) * cap), "memset");
    s->K = 0;
    dfree(s->nl);
    s->bKb = 0;
    dfree(s->bnl);
  }
  // the brick extent and window capacity follow the density
  s->brickB[0] = s->brickB[1] = s->brickB[2] = 0;
  s->brickWmax = 0;
  s->n = n;
  push_pa(s);
  copy_soa_up(s, s->A.id, h.id, 1);
  copy_soa_up(s, s->A.type, h.type, 1);
  copy_soa_up(s, s->A.mass, h.mass, 1);
  copy_soa_up(s, s->A.x, h.x, 3);
  copy_soa_up(s, s->A.v, h.v, 3);
  copy_soa_up(s, s->A.img, h.img, 3);
  std::vector<double> f = h.f;
  if (f.size() != h.x.size()) f.assign(h.x.size(), 0.0);
  copy_soa_up(s, s->ftot, f, 3);
  cuda_check(cudaMemset(s->ffix, 0, sizeof(long long) * 3 * s->cap), "memset");
  cuda_check(cudaMemset(s->f64, 0, sizeof(double) * 3 * s->cap), "memset");
  s->binned = false;
  ensure_mlp_scratch(s);
}

// Dense id map, bond and exclusion CSRs indexed by id - idMin.
void rebuild_id_tables(espp_system* s) {
  dfree(s->id2idx);
  dfree(s->bondStart);
  dfree(s->bondPartner);
  dfree(s->langExcl);
  dfree(s->halo);
  dfree(s->exclStart);
  dfree(s->exclIds);
  if (s->allIds.empty()) {
    s->idMin = 0;
    s->idSpan = 0;
    s->idDirty = false;
    return;
  }
  auto mm = std::minmax_element(s->allIds.begin(), s->allIds.end());
  s->idMin = *mm.first;
  int64_t span = *mm.second - *mm.first + 1;
  // a domain of a spatial decomposition holds a slab of the ids of the whole system
  if (span > 16 * (int64_t)s->allIds.size() + (1 << 24) || span > (1LL << 31) - 2)
    raise(ESPP_ERANGE, "particle ids are too sparse for the dense id map (span " +
                           std::to_string(span) + ")");
  s->idSpan = (int)span;
  s->id2idx = dalloc<int32_t>(span);
  cuda_check(cudaMemset(s->id2idx, 0xff, sizeof(int32_t) * span), "memset");
  auto csr = [&](const std::vector<std::pair<int64_t, int64_t>>& pairs, int32_t*& dstart,
                 int64_t*& dids) {
    std::vector<int32_t> start(span + 1, 0);
    for (auto& p : pairs) {
      start[p.first - s->idMin + 1]++;
      start[p.second - s->idMin + 1]++;
    }
    for (int64_t k = 0; k < span; ++k) start[k + 1] += start[k];
    std::vector<int64_t> ids(std::max<int64_t>(start[span], 1));
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (auto& p : pairs) {
      ids[fill[p.first - s->idMin]++] = p.second;
      ids[fill[p.second - s->idMin]++] = p.first;
    }
    dstart = dalloc<int32_t>(span + 1);
    dids = dalloc<int64_t>(ids.size());
    cuda_check(cudaMemcpy(dstart, start.data(), sizeof(int32_t) * (span + 1),
                          cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(dids, ids.data(), sizeof(int64_t) * ids.size(),
                          cudaMemcpyHostToDevice), "upload");
  };
  for (auto& b : s->bonds)
    if (b.first < s->idMin || b.second < s->idMin || b.first - s->idMin >= span ||
        b.second - s->idMin >= span)
      raise(ESPP_EINVAL, "bond partner does not exist");
  csr(s->bonds, s->bondStart, s->bondPartner);
  std::vector<std::pair<int64_t, int64_t>> ex;
  for (auto& e : s->vlExcl)
    if (e.first >= s->idMin && e.second >= s->idMin && e.first - s->idMin < span &&
        e.second - s->idMin < span)
      ex.push_back(e);
  if (!ex.empty()) csr(ex, s->exclStart, s->exclIds);
  // triples: ids and, per particle, the triples it belongs to with its role
  dfree(s->bnl);
  dfree(s->bpartials);
  dfree(s->d_triples);
  dfree(s->tripStart);
  dfree(s->tripEntry);
  dfree(s->tripF);
  if (!s->triples.empty()) {
    const size_t nt = s->triples.size();
    std::vector<int64_t> ids(3 * nt);
    std::vector<int32_t> start(span + 1, 0);
    for (size_t t = 0; t < nt; ++t)
      for (int q = 0; q < 3; ++q) {
        const int64_t id = s->triples[t][q];
        if (id < s->idMin || id - s->idMin >= span) raise(ESPP_EINVAL, "triple member does not exist");
        ids[3 * t + q] = id;
        start[id - s->idMin + 1]++;
      }
    for (int64_t k = 0; k < span; ++k) start[k + 1] += start[k];
    std::vector<int32_t> entry(3 * nt);
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (size_t t = 0; t < nt; ++t)
      for (int q = 0; q < 3; ++q) entry[fill[s->triples[t][q] - s->idMin]++] = (int32_t)(t * 4 + q);
    s->d_triples = dalloc<int64_t>(ids.size());
    s->tripStart = dalloc<int32_t>(span + 1);
    s->tripEntry = dalloc<int32_t>(entry.size());
    s->tripF = dalloc<double>(6 * nt);
    cuda_check(cudaMemcpy(s->d_triples, ids.data(), sizeof(int64_t) * ids.size(),
                          cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(s->tripStart, start.data(), sizeof(int32_t) * (span + 1),
                          cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(s->tripEntry, entry.data(), sizeof(int32_t) * entry.size(),
                          cudaMemcpyHostToDevice), "upload");
  }
  std::vector<uint8_t> le(span, 0);
  for (int64_t id : s->langExclIds)
    if (id >= s->idMin && id - s->idMin < span) le[id - s->idMin] = 1;
  s->langExcl = dalloc<uint8_t>(span);
  cuda_check(cudaMemcpy(s->langExcl, le.data(), span, cudaMemcpyHostToDevice), "upload");
  if (!s->haloIds.empty()) {
    std::vector<uint8_t> hl(span, 0);
    for (int64_t id : s->haloIds) hl[id - s->idMin] = 1;
    s->halo = dalloc<uint8_t>(span);
    cuda_check(cudaMemcpy(s->halo, hl.data(), span, cudaMemcpyHostToDevice), "upload");
  }
  s->idDirty = false;
  s->binned = false;
}

unsigned read_err(espp_system* s) {
  unsigned e = 0;
  cuda_check(cudaMemcpyAsync(&e, s->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->st),
             "error word");
  sync(s);
  return e;
}

void check_err(espp_system* s) {
  unsigned e = read_err(s);
  if (!e) return;
  cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
  if (e & kErrOutside)
    raise(ESPP_ENAN, "a particle has moved to outer space (non-finite coordinate)");
  if (e & kErrFixOverflow)
    raise(ESPP_ERANGE, "force beyond the int64 2^-32 fixed-point range (|F| >= 1e9)");
  if (e & kErrBondMissing) raise(ESPP_ESTATE, "bond partner not present");
  if (e & kErrIdRange) raise(ESPP_ESTATE, "particle id outside the id map");
  if (e & kErrNlOverflow) raise(ESPP_EOVERFLOW, "Verlet list capacity exceeded");
  if (e & kErrTimeout) raise(ESPP_ETIMEOUT, "a bounded wait inside a kernel ran out");
}

// Re-sort the particles by cell (fold = Storage::decompose semantics).
void bin(espp_system* s, bool fold) {
  if (s->idDirty) rebuild_id_tables(s);
  DevView d = s->view();
  if (s->n == 0) {
    cuda_check(cudaMemsetAsync(s->cellStart, 0, sizeof(int32_t) * (d.ncells + 1), s->st),
               "memset");
    s->binned = true;
    return;
  }
  launch_fold_bin(d, s->scr, fold, s->st);
  launch_sort_cells(d, s->scr, s->st);
  launch_gather(d, s->scr, s->st);  // gathers into pa[1] and swaps on the device
  s->paHostValid = false;
  s->xrelFresh = true;
  launch_id_map(d, s->st);
  cuda_check(cudaGetLastError(), "re-binning kernels");
  s->binned = true;
  s->listValid = false;
}

int estimate_K(espp_system* s) {
  double V = s->L[0] * s->L[1] * s->L[2];
  double rho = s->n / V;
  double rcut = s->vl_cut + s->skin;
  double expected = rho * 4.0 / 3.0 * M_PI * rcut * rcut * rcut;
  int K = (int)std::ceil(expected * 1.6) + 32;
  return (K + 7) / 8 * 8;
}

DevCounters get_counters(espp_system* s);

// Whether the list and pair kernels take the brick form: LJ (plain or capped, FENE
// bonds, exclusions) on a grid of at least 2 cells per dimension.  Tabulated pair
// potentials and the learned potential read the per-particle form.
bool pair_any(const espp_system* s);
bool brick_wanted(const espp_system* s) {
  if (!s->brickAllowed || !s->has_vl || !s->lj_any || s->tabNT > 0 || s->mlp) return false;
  if (s->hci != 1 || !s->haloIds.empty()) return false;
  for (int k = 0; k < 3; ++k)
    if (s->nc[k] < 2) return false;
  return true;
}

// Brick extent: the largest brick of at most 240 particles (the block has 256 threads,
// one per particle) and at most kBrickMax cells per edge, grown one dimension at a time.
void choose_brick(espp_system* s) {
  const double ncells = (double)s->nc[0] * s->nc[1] * s->nc[2];
  const double occ = std::max(s->n / ncells, 0.05);
  const double target = 240.0;
  int b[3] = {1, 1, 1};
  for (bool grew = true; grew;) {
    grew = false;
    for (int k = 2; k >= 0; --k) {
      if (b[k] >= std::min(kBrickMax, s->nc[k])) continue;
      const double vol = occ * (b[0] + (k == 0)) * (b[1] + (k == 1)) * (b[2] + (k == 2));
      if (vol > target) continue;
      ++b[k];
      grew = true;
    }
  }
  for (int k = 0; k < 3; ++k) s->brickB[k] = b[k];
}

int brick_window_limit(const espp_system* s) {
  (void)s;
  const int bySmem = (int)(brick_smem_limit() / (sizeof(double) * 4 + sizeof(int)));
  return std::min(65536, bySmem) / 32 * 32;
}

bool brick_geometry_ok(const espp_system* s) {
  if (s->hci != 1) return false;  // brick windows hold one cell layer
  if (!s->haloIds.empty()) return false;  // the brick kernels know no halo particles
  for (int k = 0; k < 3; ++k)
    if (s->nc[k] < 2) return false;
  return s->n > 0;
}

// Brick extent, window capacity and partial-sum rows for the current particles and grid.
void ensure_brick_window(espp_system* s) {
  if (s->brickB[0] == 0) choose_brick(s);
  if (s->brickWmax == 0) {
    double V = 1.0;
    for (int k = 0; k < 3; ++k) V *= (s->brickB[k] + 2) * (s->L[k] / s->nc[k]);
    const double rho = s->n / (s->L[0] * s->L[1] * s->L[2]);
    int ncw = (s->brickB[0] + 2) * (s->brickB[1] + 2) * (s->brickB[2] + 2);
    int w = (int)std::ceil(1.35 * rho * V) + 3 * ncw + 96;  // up to 3 spare slots a cell
    w = std::max(256, (w + 31) / 32 * 32);
    s->brickWmax = std::min(w, brick_window_limit(s));
  }
  BrickView bv = s->brick_view();
  if (bv.nbricks * 7 > s->bpartialsCap) {
    dfree(s->bpartials);
    s->bpartialsCap = bv.nbricks * 7;
    s->bpartials = dalloc<double>(s->bpartialsCap);
  }
}

// Buffers of the brick form: the window and the window-index lists.
void ensure_brick_buffers(espp_system* s) {
  ensure_brick_window(s);
  if (s->bKb == 0 || !s->bnl) {
    if (s->bKb == 0) s->bKb = estimate_K(s);
    dfree(s->bnl);
    s->bnl = dalloc<uint16_t>((size_t)s->bKb * s->cap);
  }
}

void grow_brick_lists(espp_system* s, int need) {
  s->bKb = (std::max(s->bKb * 2, need + 32) + 7) / 8 * 8;
  dfree(s->bnl);
  s->bnl = dalloc<uint16_t>((size_t)s->bKb * s->cap);
}

// Doubles the window capacity; false when it is at its limit.
bool grow_brick_window(espp_system* s) {
  const int lim = brick_window_limit(s);
  if (s->brickWmax >= lim) return false;
  s->brickWmax = std::min(lim, s->brickWmax * 2);
  return true;
}

// The per-particle global form: built by brick windows when the grid allows (every
// candidate read once per brick from shared memory), else by the per-cell lane kernel.
void build_list_plain(espp_system* s, double cutsq) {
  if (s->K == 0 || !s->nl) {
    s->K = estimate_K(s);
    dfree(s->nl);
    s->nl = dalloc<int32_t>((size_t)s->K * s->cap);
  }
  bool useBrick = s->brickBuild && brick_geometry_ok(s);
  if (useBrick) ensure_brick_window(s);
  for (int attempt = 0; attempt < 12; ++attempt) {
    DevView d = s->view();
    if (useBrick) {
      launch_build_brick(d, cutsq, s->st);
    } else {
      const bool fresh = s->xrelFresh;
      if (!fresh) launch_xrel(d, s->st);
      s->xrelFresh = false;
      launch_build_nl(d, cutsq, fresh, s->st);
    }
    cuda_check(cudaGetLastError(), "Verlet list kernel");
    unsigned e = read_err(s);
    if (!(e & (kErrNlOverflow | kErrWindow))) break;
    cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
    if (e & kErrWindow) {
      if (!grow_brick_window(s)) useBrick = false;  // too dense for the stage
      continue;
    }
    s->K *= 2;
    dfree(s->nl);
    s->nl = dalloc<int32_t>((size_t)s->K * s->cap);
  }
  s->brickBuildUsed = useBrick;
}

// Brick form; false when a window cannot be staged (the caller falls back to the
// per-particle form).
bool build_list_brick(espp_system* s, double cutsq) {
  ensure_brick_buffers(s);
  for (int attempt = 0; attempt < 8; ++attempt) {
    DevView d = s->view();
    launch_build_brick(d, cutsq, s->st);
    cuda_check(cudaGetLastError(), "brick Verlet list kernels");
    unsigned e = read_err(s);
    if (!(e & (kErrNlOverflow | kErrWindow))) return true;
    cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
    if (e & kErrWindow) {
      if (!grow_brick_window(s)) return false;
      ensure_brick_buffers(s);
    }
    if (e & kErrNlOverflow) grow_brick_lists(s, get_counters(s).nnMax);
  }
  return false;
}

void build_list(espp_system* s) {
  if (!s->has_vl) return;
  if (!s->binned) bin(s, false);
  double cutVerlet = s->vl_cut + s->skin;
  double cutsq = cutVerlet * cutVerlet;
  s->brickOn = brick_wanted(s) && s->n > 0;
  if (s->brickOn && !build_list_brick(s, cutsq)) {
    s->brickOn = false;
    s->brickAllowed = false;  // a window too dense for the stage: per-particle form from now on
  }
  if (!s->brickOn) build_list_plain(s, cutsq);
  check_err(s);
  s->builds++;
  s->listValid = true;
}

void decompose(espp_system* s) {
  bin(s, true);
  check_err(s);
  build_list(s);
}

void upload_lj(espp_system* s) {
  // the table covers every particle type present, unset pairs interact with nothing
  int nt = std::max(s->lj.ntypes, s->maxType + 1);
  s->lj.ntypes = nt;
  std::vector<LJPair> compact((size_t)nt * nt);
  for (int a = 0; a < nt; ++a)
    for (int b = 0; b < nt; ++b) compact[(size_t)a * nt + b] = s->lj.p[a * kMaxTypes + b];
  LJTable t{};
  t.ntypes = nt;
  for (size_t k = 0; k < compact.size(); ++k) t.p[k] = compact[k];
  std::vector<LJPairF> f(kMaxTypes * kMaxTypes);
  make_float_table(t, f.data());
  dfree(s->d_lj);
  dfree(s->d_ljf);
  s->d_lj = dalloc<LJPair>(std::max<size_t>(compact.size(), 1));
  s->d_ljf = dalloc<LJPairF>(std::max<size_t>(compact.size(), 1));
  cuda_check(cudaMemcpy(s->d_lj, t.p, sizeof(LJPair) * compact.size(), cudaMemcpyHostToDevice),
             "upload");
  cuda_check(cudaMemcpy(s->d_ljf, f.data(), sizeof(LJPairF) * compact.size(),
                        cudaMemcpyHostToDevice), "upload");
  s->lj.single = (nt == 1 && compact[0].set) ? 1 : 0;
}

constexpr int kTabBondKey = -1;
constexpr int kTabAngleKey = -2;

// Builds every table of the system into one coefficient array and uploads it with the
// descriptors and the type-pair map.
void upload_tabs(espp_system* s) {
  std::vector<TabDesc> descs;
  std::vector<double> coef;
  int nt = 0;
  for (auto& kv : s->tabSpecs)
    if (kv.first >= 0) nt = std::max(nt, kv.first % kMaxTypes + 1);
  nt = nt > 0 ? std::max(nt, s->maxType + 1) : 0;
  std::vector<int32_t> pairMap((size_t)nt * nt, -1);
  int bondIdx = -1, angleIdx = -1;
  for (auto& kv : s->tabSpecs) {
    const espp_system::TabSpec& t = kv.second;
    TabDesc desc;
    const char* msg = build_table(t.itype, (int)t.r.size(), t.r.data(), t.e.data(),
                                  t.f.data(), desc, coef);
    if (msg) raise(ESPP_EINVAL, msg);
    desc.rcsq = t.rc * t.rc;
    desc.shift = t.shift;
    const int idx = (int)descs.size();
    descs.push_back(desc);
    if (kv.first == kTabBondKey) {
      bondIdx = idx;
    } else if (kv.first == kTabAngleKey) {
      angleIdx = idx;
    } else {
      const int t1 = kv.first / kMaxTypes, t2 = kv.first % kMaxTypes;
      pairMap[(size_t)t1 * nt + t2] = idx;
      pairMap[(size_t)t2 * nt + t1] = idx;
    }
  }
  dfree(s->d_tabs);
  dfree(s->d_tabCoef);
  dfree(s->d_tabPair);
  if (!descs.empty()) {
    s->d_tabs = dalloc<TabDesc>(descs.size());
    s->d_tabCoef = dalloc<double>(coef.size());
    cuda_check(cudaMemcpy(s->d_tabs, descs.data(), sizeof(TabDesc) * descs.size(),
                          cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(s->d_tabCoef, coef.data(), sizeof(double) * coef.size(),
                          cudaMemcpyHostToDevice), "upload");
  }
  if (nt > 0) {
    s->d_tabPair = dalloc<int32_t>(pairMap.size());
    cuda_check(cudaMemcpy(s->d_tabPair, pairMap.data(), sizeof(int32_t) * pairMap.size(),
                          cudaMemcpyHostToDevice), "upload");
  }
  s->tabNT = nt;
  s->tabBond = bondIdx;
  s->tabAngle = angleIdx;
}

// whether a pair interaction runs on the Verlet list
bool pair_any(const espp_system* s) { return s->lj_any || s->tabNT > 0 || s->mlp; }

// per-particle buffers of the learned potential, sized to the particle capacity
void ensure_mlp_scratch(espp_system* s) {
  if (!s->mlp || s->mlpCap >= s->cap) return;
  const size_t c = (size_t)std::max(s->cap, 1);
  dfree(s->mlpG);
  dfree(s->mlpD);
  dfree(s->mlpE);
  dfree(s->mlpF);
  dfree(s->mlpErr);
  dfree(s->mlpTan);
  dfree(s->mlpPart);
  dfree(s->mlpFref);
  s->mlpG = dalloc<float>(c * kMlpK);
  s->mlpD = dalloc<float>(c * kMlpK);
  s->mlpE = dalloc<float>(c);
  s->mlpF = dalloc<float>(c * 3);
  s->mlpErr = dalloc<float>(c * 3);
  s->mlpTan = dalloc<float>(c * kMlpK);
  s->mlpPart = dalloc<float>((size_t)mlp_grad_blocks((int)c) * kMlpParams);
  s->mlpFref = dalloc<double>(c * 3);
  s->mlpCap = s->cap;
}

// Main pair + FENE kernel (list counts zeroed when no LJ pair is set), then the
// tabulated pair and bond forces added to its output.
void launch_all_forces(espp_system* s, cudaStream_t st) {
  DevView d = s->view();
  const bool mixed = s->precision == ESPP_PREC_MIXED;
  DevView dm = d;
  if (s->brickOn) {
    launch_forces_brick(d, mixed, s->fene, st);
  } else {
    if (!s->has_vl || !s->lj_any) dm.nn = s->nnZero;  // no LJ term: bonds only
    launch_forces(dm, mixed, s->fene, s->tpp, st);
  }
  if (!s->has_vl) d.tabNT = 0;
  launch_force_tab(d, mixed, st);
  if (d.mlp.on) launch_mlp_forces(d, mixed, nullptr, st);
  launch_angle_forces(d, mixed, st);
}

void forces(espp_system* s) {
  if (s->has_vl && pair_any(s) && !s->listValid) build_list(s);
  launch_all_forces(s, s->st);
}


IntegrateArgs integrate_args(espp_system* s) {
  IntegrateArgs a{};
  a.mixed = s->precision == ESPP_PREC_MIXED;
  a.dt = s->dt;
  a.langevin = s->lang_on ? 1 : 0;
  a.pref1 = -s->gamma;
  a.pref2 = std::sqrt(24.0 * s->temperature * s->gamma / s->dt);
  a.capMode = s->capMode;
  for (int k = 0; k < 3; ++k) a.cap[k] = s->cap3[k];
  a.seed = s->seed;
  return a;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// ---- device-event phase timing ---------------------------------------------------
enum { kPhForce = 0, kPhIntegrate = 1, kPhRebuild = 2, kPhOther = 3, kPhList = 4, kNumPh = 8 };

cudaEvent_t next_event(espp_system* s) {
  if (s->evUsed == s->evPool.size()) {
    cudaEvent_t e;
    cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    s->evPool.push_back(e);
  }
  return s->evPool[s->evUsed++];
}

struct PhaseScope {
  espp_system* s;
  int ph;
  size_t idx;
  PhaseScope(espp_system* s_, int ph_, int launches) : s(s_), ph(ph_) {
    s->phaseLaunches[ph] += launches;
    if (!s->profiling) return;
    idx = s->evUsed;
    cuda_check(cudaEventRecord(next_event(s), s->st), "event");
  }
  ~PhaseScope() {
    if (!s->profiling) return;
    if (cudaEventRecord(next_event(s), s->st) == cudaSuccess) s->evPhase.push_back({ph, idx});
  }
};

void collect_phases(espp_system* s) {
  if (!s->profiling) return;
  sync(s);
  for (auto& pe : s->evPhase) {
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, s->evPool[pe.second], s->evPool[pe.second + 1]),
               "event time");
    s->phaseMs[pe.first] += ms;
  }
  s->evPhase.clear();
  s->evUsed = 0;
}

// rebuild = fold/bin (fold_bin, scan, scatter, sort, gather, id map) + Verlet list
void timed_decompose(espp_system* s) {
  {
    PhaseScope ps(s, kPhRebuild, 10);
    bin(s, true);
  }
  check_err(s);
  PhaseScope ps(s, kPhList, s->has_vl ? 1 : 0);
  build_list(s);
}

void timed_forces(espp_system* s) {
  PhaseScope ps(s, kPhForce, 1);
  forces(s);
}

void timed_integrate(espp_system* s, const IntegrateArgs& a) {
  PhaseScope ps(s, kPhIntegrate, 1);
  launch_integrate(s->view(), a, s->st);
}

void set_counters(espp_system* s, const DevCounters& c) {
  *s->hctr = c;
  cuda_check(cudaMemcpyAsync(s->ctr, s->hctr, sizeof(DevCounters), cudaMemcpyHostToDevice, s->st),
             "counters");
}

DevCounters get_counters(espp_system* s) {
  cuda_check(cudaMemcpyAsync(s->hctr, s->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s->st),
             "counters");
  sync(s);
  return *s->hctr;
}

void destroy_graph(espp_system* s) {
  if (s->graphExec) cudaGraphExecDestroy(s->graphExec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graphExec = nullptr;
  s->graph = nullptr;
  s->graphKey.clear();
}

// Everything a captured launch bakes in: kernel arguments and launch shapes.
std::string graph_key(espp_system* s, const IntegrateArgs& a) {
  DevView d = s->view();
  std::string k((const char*)&d, sizeof(d));
  k.append((const char*)&a, sizeof(a));
  k.append((const char*)&s->fene, sizeof(s->fene));
  int extra[4] = {s->tpp, s->has_vl ? 1 : 0, s->lj_any ? 1 : 0, s->precision};
  k.append((const char*)extra, sizeof(extra));
  double sk = s->skin + s->vl_cut;
  k.append((const char*)&sk, sizeof(sk));
  return k;
}

// Re-sort + Verlet build launched on st (also used to populate the IF body).
void launch_rebuild_kernels(espp_system* s, cudaStream_t st) {
  DevView d = s->view();
  launch_fold_bin(d, s->scr, true, st);
  launch_sort_cells(d, s->scr, st);
  launch_gather(d, s->scr, st);
  launch_id_map(d, st);
  if (s->has_vl) {
    const double cv = s->vl_cut + s->skin;
    if (s->brickOn || s->brickBuildUsed) {
      launch_build_brick(d, cv * cv, st);  // window-index or global form (d.brick.on)
    } else {
      launch_build_nl(d, cv * cv, true, st);
    }
  }
}

void launch_force_kernel(espp_system* s, cudaStream_t st) { launch_all_forces(s, st); }

// Adds to graph g one WHILE node (no dependencies) running the step loop of s:
// WHILE(remaining) { decide; IF(re-sort) { fold, bin, sort, gather, swap, id map, list };
//                    force; integrate2 + integrate1 }
void add_step_loop(espp_system* s, cudaGraph_t g, const IntegrateArgs& ai) {
  cudaGraphConditionalHandle hWhile, hIf;
  cuda_check(cudaGraphConditionalHandleCreate(&hWhile, g, 1, cudaGraphCondAssignDefault),
             "conditional handle");
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hWhile;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  cuda_check(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp), "while node");
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  cuda_check(cudaGraphConditionalHandleCreate(&hIf, body, 0, cudaGraphCondAssignDefault),
             "conditional handle");
  cudaStream_t cs;
  cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
  // on an error inside a capture: end it and release the stream before the error leaves
  struct CaptureGuard {
    cudaStream_t cs;
    ~CaptureGuard() {
      cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(cs, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
      }
      cudaGetLastError();
      cudaStreamDestroy(cs);
    }
  } guard{cs};
  const double skinHalf = 0.5 * s->skin;
  // body: decide
  cuda_check(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal), "capture");
  launch_decide_graph(s->view(), skinHalf, hIf, hWhile, cs);
  cudaStreamCaptureStatus st;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cuda_check(cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &deps, &ndeps), "capture info");
  cudaGraphNodeParams ip = {};
  ip.type = cudaGraphNodeTypeConditional;
  ip.conditional.handle = hIf;
  ip.conditional.type = cudaGraphCondTypeIf;
  ip.conditional.size = 1;
  cudaGraphNode_t inode;
  cuda_check(cudaGraphAddNode(&inode, body, deps, ndeps, &ip), "if node");
  cuda_check(cudaStreamUpdateCaptureDependencies(cs, &inode, 1, cudaStreamSetCaptureDependencies),
             "capture dependencies");
  launch_force_kernel(s, cs);
  launch_integrate(s->view(), ai, cs);
  cudaGraph_t done;
  cuda_check(cudaStreamEndCapture(cs, &done), "end capture");
  // IF body: re-sort and list build
  cudaGraph_t rb = ip.conditional.phGraph_out[0];
  cuda_check(cudaStreamBeginCaptureToGraph(cs, rb, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal), "capture");
  launch_rebuild_kernels(s, cs);
  cuda_check(cudaStreamEndCapture(cs, &done), "end capture");
}

void capture_graph(espp_system* s, const IntegrateArgs& ai) {
  destroy_graph(s);
  cudaGraph_t g;
  cuda_check(cudaGraphCreate(&g, 0), "cudaGraphCreate");
  cudaGraphExec_t ex = nullptr;
  try {
    add_step_loop(s, g, ai);
    cuda_check(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate");
  } catch (...) {
    cudaGraphDestroy(g);
    throw;
  }
  s->graph = g;
  s->graphExec = ex;
}

void ensure_snapshot(espp_system* s) {
  if (s->snapCap >= s->cap) return;
  free_particles(s->snap);
  alloc_particles(s->snap, s->cap);
  s->snapCap = s->cap;
}

void copy_arrays(espp_system* s, const ParticleArrays& dst, const ParticleArrays& src) {
  const size_t c = s->cap;
  cuda_check(cudaMemcpyAsync(dst.x, src.x, 3 * c * sizeof(double), cudaMemcpyDeviceToDevice, s->st),
             "copy");
  cuda_check(cudaMemcpyAsync(dst.v, src.v, 3 * c * sizeof(double), cudaMemcpyDeviceToDevice, s->st),
             "copy");
  cuda_check(cudaMemcpyAsync(dst.id, src.id, c * sizeof(int64_t), cudaMemcpyDeviceToDevice, s->st),
             "copy");
  cuda_check(cudaMemcpyAsync(dst.type, src.type, c * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                             s->st), "copy");
  cuda_check(cudaMemcpyAsync(dst.mass, src.mass, c * sizeof(double), cudaMemcpyDeviceToDevice,
                             s->st), "copy");
  cuda_check(cudaMemcpyAsync(dst.img, src.img, 3 * c * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                             s->st), "copy");
}

int K_high_water(espp_system* s) { return get_counters(s).nnMax; }

// Grows the Verlet capacity ahead of need when the builds came within 10 % of it.  The
// position of an entry in either list form does not depend on the capacity (block k of
// row i sits at (k * rows + i) * 8), so the current lists are copied into the larger
// buffer and stay valid: no rebuild, which the reference would not do either.
void maybe_grow_K(espp_system* s) {
  if (!s->has_vl) return;
  const int hw = K_high_water(s);
  if (s->brickOn) {
    if (hw * 10 <= s->bKb * 9) return;
    const int Kn = (hw * 3 / 2 + 15) / 8 * 8;
    uint16_t* nl = dalloc<uint16_t>((size_t)Kn * s->cap);
    cuda_check(cudaMemcpyAsync(nl, s->bnl, sizeof(uint16_t) * (size_t)s->bKb * s->cap,
                               cudaMemcpyDeviceToDevice, s->st), "copy");
    sync(s);
    dfree(s->bnl);
    s->bnl = nl;
    s->bKb = Kn;
    return;
  }
  if (s->K == 0 || hw * 10 <= s->K * 9) return;
  const int Kn = (hw * 3 / 2 + 15) / 8 * 8;
  int32_t* nl = dalloc<int32_t>((size_t)Kn * s->cap);
  cuda_check(cudaMemcpyAsync(nl, s->nl, sizeof(int32_t) * (size_t)s->K * s->cap,
                             cudaMemcpyDeviceToDevice, s->st), "copy");
  sync(s);
  dfree(s->nl);
  s->nl = nl;
  s->K = Kn;
}

// The list form follows the interactions (brick_wanted); a list built before the
// potentials were set (espp_vl_create comes first) is rebuilt in the other form at the
// same positions, without counting a build.
void ensure_list_form(espp_system* s) {
  if (!s->has_vl || !s->listValid || s->n == 0) return;
  if (brick_wanted(s) == s->brickOn) return;
  const int64_t builds = s->builds;
  build_list(s);
  s->builds = builds;
}

// Everything of VelocityVerlet::run before the step loop (src/integrator/
// VelocityVerlet.cpp:63-103): re-sort if flagged, lists, device counters, and the
// start-of-run force with the Langevin heat-up factor followed by integrate1 of step 0.
// Returns the integrate arguments of the loop.
IntegrateArgs run_prologue(espp_system* s, int64_t nsteps, double& tResort) {
  s->nResorts = 0;
  if (!s->runBeg) {
    cuda_check(cudaEventCreate(&s->runBeg), "event");
    cuda_check(cudaEventCreate(&s->runLoop), "event");
    cuda_check(cudaEventCreate(&s->runEnd), "event");
  }
  cuda_check(cudaEventRecord(s->runBeg, s->st), "event");
  if (s->idDirty) rebuild_id_tables(s);
  if (s->resortFlag) {
    double tr = now_s();
    timed_decompose(s);
    DevCounters c = get_counters(s);
    c.maxDist = 0.0;
    set_counters(s, c);
    s->resortFlag = false;
    tResort += now_s() - tr;
  }
  if (!s->binned) bin(s, false);
  if (s->has_vl && !s->listValid) build_list(s);
  ensure_list_form(s);
  IntegrateArgs a = integrate_args(s);
  DevCounters c0 = get_counters(s);
  c0.maxSq = 0ull;
  c0.resorts = 0;
  c0.step = s->step - 1;
  c0.remaining = nsteps;
  c0.pref1 = a.pref1;
  c0.pref2 = a.pref2;
  set_counters(s, c0);
  // start-of-run force (recalc1 = heatUp: pref2 * sqrt(3); recalc2 restores it)
  timed_forces(s);
  IntegrateArgs a0 = a;
  a0.pref2 = a.pref2 * std::sqrt(3.0);
  a0.phase = 1;
  a0.step = s->step;
  a0.do_i2 = 0;
  a0.do_i1 = nsteps > 0 ? 1 : 0;
  a0.storeFtot = nsteps > 0 ? 0 : 1;
  timed_integrate(s, a0);
  cuda_check(cudaGetLastError(), "start-of-run kernels");
  cuda_check(cudaEventRecord(s->runLoop, s->st), "event");
  IntegrateArgs ai = a;
  ai.phase = 0;
  ai.do_i2 = 1;
  ai.do_i1 = 1;
  ai.storeFtot = 0;
  return ai;
}

// Arguments baked into a captured step loop: step and Langevin prefactors come from
// the device counters.
IntegrateArgs graph_args(const IntegrateArgs& ai) {
  IntegrateArgs ag = ai;
  ag.fromCounters = 1;
  ag.step = 0;
  ag.pref1 = 0.0;
  ag.pref2 = 0.0;
  return ag;
}

void run_host_loop(espp_system* s, int64_t nsteps, const IntegrateArgs& ai, double& tResort) {
  const double skinHalf = 0.5 * s->skin;
  for (int64_t i = 0; i < nsteps; ++i) {
    {
      PhaseScope ps(s, kPhOther, 1);
      launch_decide(s->view(), skinHalf, s->st);
    }
    cuda_check(cudaMemcpyAsync(s->hctr, s->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                               s->st), "flag");
    sync(s);
    if (s->hctr->flag) {
      double tr = now_s();
      timed_decompose(s);
      s->nResorts++;
      tResort += now_s() - tr;
    }
    timed_forces(s);
    IntegrateArgs aj = ai;
    aj.step = s->step;
    aj.do_i1 = (i + 1 < nsteps) ? 1 : 0;
    aj.storeFtot = (i + 1 < nsteps) ? 0 : 1;
    timed_integrate(s, aj);
    cuda_check(cudaGetLastError(), "step kernels");
    s->step++;
  }
  cuda_check(cudaEventRecord(s->runEnd, s->st), "event");
}

// Bookkeeping after a graph-run step loop of nsteps.
void graph_loop_done(espp_system* s, int64_t nsteps) {
  DevCounters c = get_counters(s);
  s->step += nsteps;
  s->nResorts = c.resorts;
  s->builds += c.resorts;
  // kernels launched by the graph: decide + force + integrate per step, and zero,
  // fold/bin, scan (3), scatter, in-cell sort, gather, swap, id map (+ list) per re-sort
  s->phaseLaunches[kPhOther] += nsteps;
  s->phaseLaunches[kPhForce] += nsteps;
  s->phaseLaunches[kPhIntegrate] += nsteps;
  s->phaseLaunches[kPhRebuild] += c.resorts * 10;
  s->phaseLaunches[kPhList] += s->has_vl ? c.resorts : 0;
  s->paHostValid = false;
}

void run_epilogue(espp_system* s, double t0, double tResort, bool graphDone) {
  sync(s);
  check_err(s);
  maybe_grow_K(s);
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, s->runBeg, s->runEnd), "event time");
  s->lastRunMs = ms;
  cuda_check(cudaEventElapsedTime(&ms, s->runLoop, s->runEnd), "event time");
  s->lastLoopMs = ms;
  collect_phases(s);
  const double t1 = now_s();
  s->timers[0] = t1 - t0;
  s->timers[1] = s->phaseMs[kPhForce] * 1e-3;
  s->timers[6] = s->phaseMs[kPhIntegrate] * 1e-3;
  s->timers[8] = graphDone ? (s->phaseMs[kPhRebuild] + s->phaseMs[kPhList]) * 1e-3 : tResort;
  s->timers[9] = s->timers[0] - s->timers[1] - s->timers[6] - s->timers[8];
}

// State at the start of a graph run, kept so that a Verlet-list overflow inside the
// graph can be undone: particle arrays (copied on the device) and the host counters.
struct RunSnapshot {
  DevCounters ctr;
  int64_t step, builds;
  bool resortFlag;
};

RunSnapshot take_snapshot(espp_system* s) {
  sync_pa(s);
  ensure_snapshot(s);
  copy_arrays(s, s->snap, s->A);
  RunSnapshot r;
  r.ctr = get_counters(s);
  r.step = s->step;
  r.builds = s->builds;
  r.resortFlag = s->resortFlag;
  return r;
}

// Restores the state saved before a graph run whose Verlet list overflowed and grows the
// list capacity (the caller then redoes the run on the host loop).  The list is rebuilt
// at the restored positions without counting a build: the accumulated displacement is
// restored too, so re-sorts and builds fall on the same steps as in a run that never
// overflowed, and the new list holds every pair the old one held within the cutoff
// until the next re-sort.
void recover_overflow(espp_system* s, const RunSnapshot& r) {
  const int hw = K_high_water(s);  // the graph's largest count, before the restore
  const unsigned why = read_err(s);
  cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
  s->paHostValid = false;
  sync_pa(s);
  copy_arrays(s, s->A, s->snap);
  set_counters(s, r.ctr);
  s->step = r.step;
  s->resortFlag = r.resortFlag;
  s->binned = false;
  if (why & kErrWindow) {
    if (!grow_brick_window(s)) {  // too dense for the stage: no brick kernels from now on
      s->brickOn = false;
      s->brickAllowed = false;
      s->brickBuild = false;
    }
  } else if (s->brickOn) {
    grow_brick_lists(s, hw);
  } else {
    s->K = (std::max(s->K * 2, hw + 32) + 7) / 8 * 8;  // multiple of 8
    dfree(s->nl);
    s->nl = dalloc<int32_t>((size_t)s->K * s->cap);
  }
  s->listValid = false;
  destroy_graph(s);
  if (!s->resortFlag) {
    bin(s, false);
    build_list(s);
  }
  s->builds = r.builds;
}

void run_host(espp_system* s, int64_t nsteps);

// VelocityVerlet::run (src/integrator/VelocityVerlet.cpp:63-169).
void run(espp_system* s, int64_t nsteps) {
  if (!(nsteps > 0 && s->useGraph && !s->profiling)) {
    run_host(s, nsteps);
    return;
  }
  const double t0 = now_s();
  double tResort = 0.0;
  RunSnapshot snap = take_snapshot(s);
  IntegrateArgs ai = run_prologue(s, nsteps, tResort);
  IntegrateArgs ag = graph_args(ai);
  std::string key = graph_key(s, ag);
  if (!s->graphExec || key != s->graphKey) {
    capture_graph(s, ag);
    s->graphKey = key;
  }
  cuda_check(cudaGraphLaunch(s->graphExec, s->st), "cudaGraphLaunch");
  cuda_check(cudaEventRecord(s->runEnd, s->st), "event");
  sync(s);
  if (read_err(s) & (kErrNlOverflow | kErrWindow)) {
    // back to the state before the run, a larger list, and the run again on the host loop
    recover_overflow(s, snap);
    run_host(s, nsteps);
    return;
  }
  graph_loop_done(s, nsteps);
  run_epilogue(s, t0, tResort, true);
}

void run_host(espp_system* s, int64_t nsteps) {
  const double t0 = now_s();
  double tResort = 0.0;
  IntegrateArgs ai = run_prologue(s, nsteps, tResort);
  run_host_loop(s, nsteps, ai, tResort);
  run_epilogue(s, t0, tResort, false);
}

}  // namespace

// Many independent systems stepped by one graph launch: one WHILE branch per system, no
// dependencies between the branches, so the GPU runs the replicas' kernels concurrently
// and each keeps its own re-sort schedule (ParallelTempering / MultiSystem,
// src/ParallelTempering.py:78-203, src/MultiSystem.py:105-125).
struct espp_batch {
  std::vector<espp_system*> sys;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  std::string key;
  cudaEvent_t beg = nullptr, end = nullptr;
  std::vector<cudaEvent_t> ready;
  double lastMs = 0.0;
};

namespace {

void batch_destroy_graph(espp_batch* b) {
  if (b->ex) cudaGraphExecDestroy(b->ex);
  if (b->g) cudaGraphDestroy(b->g);
  b->ex = nullptr;
  b->g = nullptr;
  b->key.clear();
}

void batch_run(espp_batch* b, int64_t nsteps) {
  if (nsteps <= 0) {
    for (espp_system* s : b->sys) run(s, nsteps);
    return;
  }
  const size_t R = b->sys.size();
  const double t0 = now_s();
  std::vector<RunSnapshot> snaps(R);
  std::vector<double> tRes(R, 0.0);
  std::vector<IntegrateArgs> ags(R);
  std::string key;
  for (size_t r = 0; r < R; ++r) {
    espp_system* s = b->sys[r];
    snaps[r] = take_snapshot(s);
    ags[r] = graph_args(run_prologue(s, nsteps, tRes[r]));
    key += graph_key(s, ags[r]);
    cuda_check(cudaEventRecord(b->ready[r], s->st), "event");
    cuda_check(cudaStreamWaitEvent(b->st, b->ready[r], 0), "stream wait");
  }
  if (!b->ex || key != b->key) {
    batch_destroy_graph(b);
    cuda_check(cudaGraphCreate(&b->g, 0), "cudaGraphCreate");
    try {
      for (size_t r = 0; r < R; ++r) add_step_loop(b->sys[r], b->g, ags[r]);
      cuda_check(cudaGraphInstantiate(&b->ex, b->g, 0), "cudaGraphInstantiate");
    } catch (...) {
      batch_destroy_graph(b);
      throw;
    }
    b->key = key;
  }
  cuda_check(cudaEventRecord(b->beg, b->st), "event");
  cuda_check(cudaGraphLaunch(b->ex, b->st), "cudaGraphLaunch");
  cuda_check(cudaEventRecord(b->end, b->st), "event");
  for (size_t r = 0; r < R; ++r) cuda_check(cudaEventRecord(b->sys[r]->runEnd, b->st), "event");
  cuda_check(cudaStreamSynchronize(b->st), "stream synchronize");
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, b->beg, b->end), "event time");
  b->lastMs = ms;
  for (size_t r = 0; r < R; ++r) {
    espp_system* s = b->sys[r];
    if (read_err(s) & (kErrNlOverflow | kErrWindow)) {
      recover_overflow(s, snaps[r]);
      run_host(s, nsteps);
      continue;
    }
    graph_loop_done(s, nsteps);
    run_epilogue(s, t0, tRes[r], true);
  }
}

double* obs_partials(espp_system* s, int& nb) {
  nb = observable_blocks(s->n);
  if (nb * 7 > s->partialsCap) {
    dfree(s->partials);
    s->partialsCap = nb * 7;
    s->partials = dalloc<double>(s->partialsCap);
  }
  return s->partials;
}

void prepare_observables(espp_system* s) {
  if (s->idDirty) rebuild_id_tables(s);
  if (!s->binned) bin(s, false);
  if (s->has_vl && !s->listValid) build_list(s);
  ensure_list_form(s);
}

void observable(espp_system* s, int which, int energy, double out[7]) {
  prepare_observables(s);
  for (int k = 0; k < 7; ++k) out[k] = 0.0;
  if (s->n == 0) return;
  int nb;
  double* part = obs_partials(s, nb);
  DevView d = s->view();
  if (which == ESPP_IA_LJ) {
    if (!s->has_vl || !s->lj_any) return;
    if (s->brickOn)
      launch_lj_observables_brick(d, s->bpartials, 0, s->obs, energy, s->st);
    else
      launch_lj_observables(d, part, nb, s->obs, energy, s->st);
  } else if (which == ESPP_IA_FENE) {
    if (!s->fene.on) return;
    launch_fene_observables(d, s->fene, part, nb, s->obs, energy, s->st);
  } else if (which == ESPP_IA_TAB_PAIR) {
    if (!s->has_vl || s->tabNT == 0) return;
    launch_tab_observables(d, 0, part, nb, s->obs, energy, s->st);
  } else if (which == ESPP_IA_TAB_BOND) {
    if (s->tabBond < 0) return;
    launch_tab_observables(d, 1, part, nb, s->obs, energy, s->st);
  } else if (!s->haloIds.empty() &&
             (which == ESPP_IA_COSINE || which == ESPP_IA_TAB_ANGLE || which == ESPP_IA_MLP)) {
    raise(ESPP_EINVAL, "angle and learned-potential observables are not available with halo "
                       "particles (spatial decomposition)");
  } else if (which == ESPP_IA_COSINE) {
    if (s->triples.empty() || !s->cosine.on) return;
    launch_angle_observables(d, part, nb, s->obs, energy, 0, s->st);
  } else if (which == ESPP_IA_TAB_ANGLE) {
    if (s->triples.empty() || s->tabAngle < 0) return;
    launch_angle_observables(d, part, nb, s->obs, energy, 1, s->st);
  } else if (which == ESPP_IA_MLP) {
    if (!d.mlp.on) return;
    if (!energy) raise(ESPP_EINVAL, "the virial of the learned potential is not available");
    launch_mlp_energy_terms(d, s->st);
    launch_sum_site_energy(d, part, nb, s->obs, s->st);
  } else {
    raise(ESPP_EINVAL, "unknown interaction kind");
  }
  cuda_check(cudaGetLastError(), "observable kernels");
  cuda_check(cudaMemcpyAsync(out, s->obs, sizeof(double) * 7, cudaMemcpyDeviceToHost, s->st),
             "download");
  sync(s);
}

espp_system* checked(espp_system* s) {
  if (!s) raise(ESPP_EINVAL, "null system handle");
  cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
  return s;
}

template <class F>
int guard(F&& f) {
  try {
    f();
    return ESPP_OK;
  } catch (const Fail& e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return ESPP_ENOMEM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return ESPP_EINVAL;
  }
}

void destroy(espp_system* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  free_buffers(s);
  dfree(s->cellStart);
  dfree(s->scr.cellCount);
  dfree(s->scr.tileSum);
  dfree(s->id2idx);
  dfree(s->bondStart);
  dfree(s->bondPartner);
  dfree(s->langExcl);
  dfree(s->halo);
  dfree(s->exclStart);
  dfree(s->exclIds);
  dfree(s->err);
  destroy_graph(s);
  free_particles(s->snap);
  dfree(s->ctr);
  dfree(s->d_pa);
  dfree(s->obs);
  dfree(s->partials);
  dfree(s->d_lj);
  dfree(s->d_ljf);
  dfree(s->d_tabs);
  dfree(s->d_tabCoef);
  dfree(s->d_tabPair);
  dfree(s->mlpG);
  dfree(s->mlpD);
  dfree(s->mlpE);
  dfree(s->mlpF);
  dfree(s->mlpErr);
  dfree(s->mlpTan);
  dfree(s->mlpPart);
  dfree(s->mlpFref);
  dfree(s->facc);
  dfree(s->d_triples);
  dfree(s->tripStart);
  dfree(s->tripEntry);
  dfree(s->tripF);
  dfree(s->stIds);
  dfree(s->stPos);
  dfree(s->stVel);
  dfree(s->stF);
  dfree(s->stImg);
  for (cudaEvent_t e : s->evPool) cudaEventDestroy(e);
  if (s->runBeg) cudaEventDestroy(s->runBeg);
  if (s->runLoop) cudaEventDestroy(s->runLoop);
  if (s->runEnd) cudaEventDestroy(s->runEnd);
  if (s->hctr) cudaFreeHost(s->hctr);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

}  // namespace

namespace {

// ---- allocation-free energy ------------------------------------------------------
// Scratch of espp_energy_noalloc: slots [0, 8) take the final sums, slots [8, ...) one
// row of 7 partial sums per reduction block (256 particles).  Statically sized, so
// the call never allocates; every GPU that loads this library holds these 1.8 MB
// until the process exits.
constexpr int kNoAllocMaxBlocks = 32768;
constexpr long long kNoAllocMaxParticles = (long long)kNoAllocMaxBlocks * 256;
static __device__ __align__(256) double g_noalloc_scratch[8 + 7 * kNoAllocMaxBlocks];

// Device address of g_noalloc_scratch per device, looked up with that device current
// (the host-side name of the array is only a stand-in, not a device address).  The
// address belongs to the context the module was loaded into: a caller that resets the
// device or releases and retains its primary context gets the module loaded again,
// possibly elsewhere.  So each cached address is stored with the unique id of the
// context it was looked up in (cuCtxGetId) and looked up again when the current
// context's id differs.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[256] = {nullptr};
unsigned long long g_noalloc_ctx[256] = {0};

unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
        q0 != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f0 || !f1) {
      cudaGetLastError();
      raise(ESPP_ECUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
    }
    get_current = (CtxGetCurrentFn)f0;
    get_id = (CtxGetIdFn)f1;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    raise(ESPP_ECUDA, "no current CUDA context for the energy scratch lookup");
  return id;
}

double* noalloc_scratch(int device) {
  if (device < 0 || device >= 256) raise(ESPP_ERANGE, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  const unsigned long long ctx = current_context_id();
  if (!g_noalloc_addr[device] || g_noalloc_ctx[device] != ctx) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      raise(ESPP_ECUDA, std::string("cudaGetSymbolAddress of the energy scratch failed: ") +
                            cudaGetErrorString(e));
    }
    g_noalloc_addr[device] = (double*)ptr;
    g_noalloc_ctx[device] = ctx;
  }
  return g_noalloc_addr[device];
}

}  // namespace

extern "C" {

int espp_abi_version(void) { return 1; }

size_t espp_last_error(char* buf, size_t cap) {
  if (buf && cap) {
    size_t n = std::min(cap - 1, g_err.size());
    std::memcpy(buf, g_err.data(), n);
    buf[n] = 0;
  }
  return g_err.size();
}

int espp_system_create(const double box[3], double skin, const int32_t cell_grid[3],
                       int32_t precision, uint64_t seed, espp_system** out) {
  return guard([&] {
    if (!box || !cell_grid || !out) raise(ESPP_EINVAL, "null argument");
    for (int i = 0; i < 3; ++i) {
      if (!(box[i] > 0)) raise(ESPP_EINVAL, "box lengths must be positive");
      if (cell_grid[i] <= 0) raise(ESPP_EINVAL, "cell grid dimensions have to be positive");
      if (cell_grid[i] < 3)
        raise(ESPP_ERANGE,
              "the GPU storage needs at least 3 cells per dimension (box >= 3 (cutoff + skin))");
    }
    if (precision != ESPP_PREC_FP64 && precision != ESPP_PREC_MIXED)
      raise(ESPP_EINVAL, "unknown precision mode");
    int ndev = 0;
    cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (ndev <= 0) raise(ESPP_ECUDA, "no CUDA device");
    std::unique_ptr<espp_system> s(new espp_system());
    cuda_check(cudaGetDevice(&s->device), "cudaGetDevice");
    for (int i = 0; i < 3; ++i) {
      s->L[i] = box[i];
      s->nc[i] = cell_grid[i];
    }
    s->skin = skin;
    s->precision = precision;
    s->seed = seed;
    cuda_check(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking), "stream");
    const long long ncells = (long long)cell_grid[0] * cell_grid[1] * cell_grid[2];
    if (ncells > (1LL << 30)) raise(ESPP_ERANGE, "cell grid too large");
    s->cellStart = dalloc<int32_t>(ncells + 1);
    s->scr.cellCount = dalloc<int32_t>(ncells);
    s->scr.tileSum = dalloc<int32_t>(scan_tiles((int)ncells) + 1);
    cuda_check(cudaMemset(s->cellStart, 0, sizeof(int32_t) * (ncells + 1)), "memset");
    s->err = dalloc<unsigned>(1);
    s->ctr = dalloc<DevCounters>(1);
    s->d_pa = dalloc<ParticleArrays>(2);
    s->obs = dalloc<double>(8);
    cuda_check(cudaMemset(s->err, 0, sizeof(unsigned)), "memset");
    cuda_check(cudaMemset(s->ctr, 0, sizeof(DevCounters)), "memset");
    cuda_check(cudaMemset(s->d_pa, 0, 2 * sizeof(ParticleArrays)), "memset");
    cuda_check(cudaMallocHost(&s->hctr, sizeof(DevCounters)), "pinned counters");
    if (const char* g = std::getenv("ESPP_B200_GRAPH")) s->useGraph = std::atoi(g) != 0;
    if (const char* b = std::getenv("ESPP_B200_BRICK")) s->brickAllowed = std::atoi(b) != 0;
    if (const char* b = std::getenv("ESPP_B200_BRICK_BUILD")) s->brickBuild = std::atoi(b) != 0;
    if (const char* t = std::getenv("ESPP_B200_TPP")) {
      const int v = std::atoi(t);
      if (v == 1 || v == 2 || v == 4 || v == 8) s->tpp = v;
    }
    s->lj.ntypes = 1;
    upload_lj(s.get());
    *out = s.release();
  });
}

int espp_system_destroy(espp_system* s) {
  return guard([&] { destroy(s); });
}

int espp_set_skin(espp_system* s, double skin) {
  return guard([&] {
    checked(s)->skin = skin;
  });
}

int espp_add_particles(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                       const double* mass, const double* pos, const double* vel) {
  return guard([&] {
    checked(s);
    if (n < 0 || (n > 0 && (!id || !pos))) raise(ESPP_EINVAL, "bad particle arrays");
    if (n == 0) return;
    if ((int64_t)s->n + n > (1LL << 30)) raise(ESPP_ERANGE, "too many particles");
    HostParticles h = download(s, true);
    std::unordered_map<int64_t, int> seen;
    seen.reserve(h.id.size() + n);
    for (size_t k = 0; k < h.id.size(); ++k) seen[h.id[k]] = 1;
    const double L[3] = {s->L[0], s->L[1], s->L[2]};
    for (int64_t i = 0; i < n; ++i) {
      if (seen.count(id[i])) raise(ESPP_EINVAL, "duplicate particle id " + std::to_string(id[i]));
      seen[id[i]] = 1;
      int ty = type ? type[i] : 0;
      if (ty < 0 || ty >= kMaxTypes) raise(ESPP_ERANGE, "particle type out of range [0, 8)");
      h.id.push_back(id[i]);
      h.type.push_back(ty);
      s->maxType = std::max(s->maxType, ty);
      h.mass.push_back(mass ? mass[i] : 1.0);
      for (int k = 0; k < 3; ++k) {
        // Storage::addParticle folds the position (OrthorhombicBC::foldCoordinate)
        double x = pos[3 * i + k];
        int tmp = static_cast<int>(std::floor(x * (1.0 / L[k])));
        x -= tmp * L[k];
        h.x.push_back(x);
        h.img.push_back(tmp);
        h.v.push_back(vel ? vel[3 * i + k] : 0.0);
        h.f.push_back(0.0);
      }
      s->allIds.push_back(id[i]);
    }
    upload(s, h);
    upload_lj(s);
    s->idDirty = true;
    s->resortFlag = true;
    s->K = 0;
    dfree(s->nl);
  });
}

int espp_decompose(espp_system* s) {
  return guard([&] {
    checked(s);
    decompose(s);
    DevCounters c = get_counters(s);
    c.maxDist = 0.0;
    set_counters(s, c);
    sync(s);
    s->resortFlag = false;
  });
}

int espp_num_particles(espp_system* s, int64_t* n) {
  return guard([&] { *n = checked(s)->n; });
}

void ensure_stage(espp_system* s, int64_t n) {
  if (n <= s->stageCap) return;
  dfree(s->stIds);
  dfree(s->stPos);
  dfree(s->stVel);
  dfree(s->stF);
  dfree(s->stImg);
  int cap = (int)std::max<int64_t>(n, 1024);
  s->stIds = dalloc<int64_t>(cap);
  s->stPos = dalloc<double>(3 * (size_t)cap);
  s->stVel = dalloc<double>(3 * (size_t)cap);
  s->stF = dalloc<double>(3 * (size_t)cap);
  s->stImg = dalloc<int32_t>(3 * (size_t)cap);
  s->stageCap = cap;
}

// id map valid and current particle order fixed
void ensure_id_map(espp_system* s) {
  if (s->idDirty) rebuild_id_tables(s);
  if (!s->binned) bin(s, false);
}

int espp_get_particles(espp_system* s, int64_t n, const int64_t* ids, double* pos,
                       double* vel, double* force, int32_t* image) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids) raise(ESPP_EINVAL, "null id array");
    ensure_id_map(s);
    ensure_stage(s, n);
    cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                               s->st), "upload ids");
    launch_get_by_id(s->view(), (int)n, s->stIds, pos ? s->stPos : nullptr,
                     vel ? s->stVel : nullptr, force ? s->stF : nullptr,
                     image ? s->stImg : nullptr, s->st);
    if (pos)
      cuda_check(cudaMemcpyAsync(pos, s->stPos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                                 s->st), "download");
    if (vel)
      cuda_check(cudaMemcpyAsync(vel, s->stVel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                                 s->st), "download");
    if (force)
      cuda_check(cudaMemcpyAsync(force, s->stF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                                 s->st), "download");
    if (image)
      cuda_check(cudaMemcpyAsync(image, s->stImg, sizeof(int32_t) * 3 * n,
                                 cudaMemcpyDeviceToHost, s->st), "download");
    unsigned e = read_err(s);
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
  });
}

int espp_set_particles(espp_system* s, int64_t n, const int64_t* ids, const double* pos,
                       const double* vel) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids) raise(ESPP_EINVAL, "null id array");
    ensure_id_map(s);
    ensure_stage(s, n);
    cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                               s->st), "upload ids");
    if (pos)
      cuda_check(cudaMemcpyAsync(s->stPos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice,
                                 s->st), "upload");
    if (vel)
      cuda_check(cudaMemcpyAsync(s->stVel, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice,
                                 s->st), "upload");
    launch_set_by_id(s->view(), (int)n, s->stIds, pos ? s->stPos : nullptr,
                     vel ? s->stVel : nullptr, nullptr, s->st);
    unsigned e = read_err(s);
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
    // new positions: the reference re-sorts before the next force evaluation
    if (pos) s->resortFlag = true;
  });
}

int espp_set_images(espp_system* s, int64_t n, const int64_t* ids, const int32_t* img) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids || !img) raise(ESPP_EINVAL, "null id or image array");
    ensure_id_map(s);
    ensure_stage(s, n);
    cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                               s->st), "upload ids");
    cuda_check(cudaMemcpyAsync(s->stImg, img, sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice,
                               s->st), "upload");
    launch_set_by_id(s->view(), (int)n, s->stIds, nullptr, nullptr, s->stImg, s->st);
    unsigned e = read_err(s);
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
  });
}

int espp_set_profiling(espp_system* s, int32_t on) {
  return guard([&] {
    checked(s)->profiling = on != 0;
    for (int k = 0; k < kNumPh; ++k) {
      s->phaseMs[k] = 0.0;
      s->phaseLaunches[k] = 0;
    }
  });
}

int espp_profile(espp_system* s, double ms[8], int64_t launches[8]) {
  return guard([&] {
    checked(s);
    for (int k = 0; k < kNumPh; ++k) {
      if (ms) ms[k] = s->phaseMs[k];
      if (launches) launches[k] = s->phaseLaunches[k];
    }
  });
}

int espp_last_run_ms(espp_system* s, double ms[2]) {
  return guard([&] {
    ms[0] = checked(s)->lastRunMs;
    ms[1] = s->lastLoopMs;
  });
}

int espp_select_device(int32_t device) {
  return guard([&] { cuda_check(cudaSetDevice(device), "cudaSetDevice"); });
}

int espp_vl_create(espp_system* s, double cutoff, int64_t nexcl, const int64_t* excl) {
  return guard([&] {
    checked(s);
    if (!(cutoff > 0)) raise(ESPP_EINVAL, "Verlet list cutoff must be positive");
    double cs = cutoff + s->skin;
    for (int k = 0; k < 3; ++k)
      if (s->L[k] / s->nc[k] < cs && s->L[k] < 3 * cs)
        raise(ESPP_ERANGE, "box smaller than 3 (cutoff + skin) in a dimension");
    s->has_vl = true;
    s->vl_cut = cutoff;
    for (int64_t i = 0; i < nexcl; ++i) s->vlExcl.push_back({excl[2 * i], excl[2 * i + 1]});
    if (nexcl > 0) s->idDirty = true;
    s->K = 0;
    dfree(s->nl);
    s->bKb = 0;
    dfree(s->bnl);
    if (s->idDirty) rebuild_id_tables(s);
    if (!s->binned) bin(s, false);
    build_list(s);
  });
}

int espp_vl_rebuild(espp_system* s) {
  return guard([&] {
    checked(s);
    if (!s->has_vl) raise(ESPP_ESTATE, "no Verlet list");
    if (s->idDirty) rebuild_id_tables(s);
    build_list(s);
  });
}

int espp_vl_size(espp_system* s, int64_t* npairs) {
  return guard([&] {
    checked(s);
    *npairs = 0;
    if (!s->has_vl || s->n == 0) return;
    DevView d = s->view();
    int32_t* counts = dalloc<int32_t>(s->n);
    if (s->brickOn)
      launch_pair_count_brick(d, counts, s->st);
    else
      launch_pair_count(d, counts, s->st);
    std::vector<int32_t> h(s->n);
    cudaError_t e = cudaMemcpyAsync(h.data(), counts, sizeof(int32_t) * s->n,
                                    cudaMemcpyDeviceToHost, s->st);
    cudaStreamSynchronize(s->st);
    dfree(counts);
    cuda_check(e, "download");
    int64_t t = 0;
    for (int32_t c : h) t += c;
    *npairs = t;
  });
}

int espp_vl_digest(espp_system* s, uint64_t out[4]) {
  return guard([&] {
    checked(s);
    if (!out) raise(ESPP_EINVAL, "null output pointer");
    for (int k = 0; k < 4; ++k) out[k] = 0;
    if (!s->has_vl || s->n == 0) return;
    int nb;
    // the observable partials hold 7 doubles per block; the digest needs 4 words
    unsigned long long* part = reinterpret_cast<unsigned long long*>(obs_partials(s, nb));
    unsigned long long* res = reinterpret_cast<unsigned long long*>(s->obs);
    if (s->brickOn)
      launch_pair_digest_brick(s->view(), reinterpret_cast<unsigned long long*>(s->bpartials),
                               res, s->st);
    else
      launch_pair_digest(s->view(), part, nb, res, s->st);
    cuda_check(cudaGetLastError(), "digest kernels");
    cuda_check(cudaMemcpyAsync(out, res, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->st),
               "download");
    sync(s);
  });
}

int espp_vl_pairs(espp_system* s, int64_t capn, int64_t* pairs, int64_t* npairs) {
  return guard([&] {
    checked(s);
    *npairs = 0;
    if (!s->has_vl || s->n == 0) return;
    DevView d = s->view();
    int32_t* counts = dalloc<int32_t>(s->n);
    if (s->brickOn)
      launch_pair_count_brick(d, counts, s->st);
    else
      launch_pair_count(d, counts, s->st);
    std::vector<int32_t> h(s->n);
    cuda_check(cudaMemcpyAsync(h.data(), counts, sizeof(int32_t) * s->n,
                               cudaMemcpyDeviceToHost, s->st), "download");
    sync(s);
    std::vector<int64_t> off(s->n);
    int64_t t = 0;
    for (int i = 0; i < s->n; ++i) {
      off[i] = t;
      t += h[i];
    }
    int64_t* doff = dalloc<int64_t>(s->n);
    int64_t* dout = dalloc<int64_t>(2 * std::max<int64_t>(t, 1));
    std::vector<int64_t> out(2 * std::max<int64_t>(t, 1));
    cudaMemcpy(doff, off.data(), sizeof(int64_t) * s->n, cudaMemcpyHostToDevice);
    if (s->brickOn)
      launch_pair_write_brick(d, doff, counts, dout, s->st);
    else
      launch_pair_write(d, doff, dout, s->st);
    cudaError_t e = cudaMemcpyAsync(out.data(), dout, sizeof(int64_t) * 2 * t,
                                    cudaMemcpyDeviceToHost, s->st);
    cudaStreamSynchronize(s->st);
    dfree(counts);
    dfree(doff);
    dfree(dout);
    cuda_check(e, "download");
    std::vector<std::pair<int64_t, int64_t>> v(t);
    for (int64_t k = 0; k < t; ++k) v[k] = {out[2 * k], out[2 * k + 1]};
    std::sort(v.begin(), v.end());
    *npairs = t;
    for (int64_t k = 0; k < std::min(capn, t); ++k) {
      pairs[2 * k] = v[k].first;
      pairs[2 * k + 1] = v[k].second;
    }
  });
}

int espp_vl_builds(espp_system* s, int64_t* builds) {
  return guard([&] { *builds = checked(s)->builds; });
}

int espp_lj_set(espp_system* s, int32_t t1, int32_t t2, double eps, double sig, double rc,
                double shift, double caprad) {
  return guard([&] {
    checked(s);
    if (t1 < 0 || t2 < 0 || t1 >= kMaxTypes || t2 >= kMaxTypes)
      raise(ESPP_ERANGE, "particle type out of range [0, 8)");
    LJPair P{};
    P.set = 1;
    double sig2 = sig * sig;
    double sig6 = sig2 * sig2 * sig2;
    P.ff1 = 48.0 * eps * sig6 * sig6;
    P.ff2 = 24.0 * eps * sig6;
    P.ef1 = 4.0 * eps;
    P.ef2 = sig * sig;
    P.rcsq = rc * rc;
    P.shift = shift;
    P.caprad = caprad;
    if (caprad > 0) {
      double frac2 = (sig / caprad) * (sig / caprad);
      double frac6 = frac2 * frac2 * frac2;
      P.capff = 48.0 * eps * frac6 * (frac6 - 0.5) / caprad;
    }
    s->lj.p[t1 * kMaxTypes + t2] = P;
    s->lj.p[t2 * kMaxTypes + t1] = P;
    s->lj.ntypes = std::max(s->lj.ntypes, std::max(t1, t2) + 1);
    s->lj_any = true;
    upload_lj(s);
  });
}

int espp_bonds_add(espp_system* s, int64_t n, const int64_t* pairs) {
  return guard([&] {
    checked(s);
    std::unordered_map<int64_t, int> have;
    for (int64_t id : s->allIds) have[id] = 1;
    for (int64_t i = 0; i < n; ++i) {
      int64_t a = pairs[2 * i], b = pairs[2 * i + 1];
      if (a > b) std::swap(a, b);
      if (!have.count(a) || !have.count(b)) raise(ESPP_EINVAL, "bond partner does not exist");
      s->bonds.push_back({a, b});
    }
    s->idDirty = true;
  });
}

int espp_bonds_size(espp_system* s, int64_t* n) {
  return guard([&] { *n = (int64_t)checked(s)->bonds.size(); });
}

// FixedPairList::remove (FixedPairList.cpp:317-324): the list is emptied.
int espp_bonds_clear(espp_system* s) {
  return guard([&] {
    checked(s)->bonds.clear();
    s->idDirty = true;
  });
}

int espp_fene_set(espp_system* s, double K, double r0, double rmax, double rc, double shift) {
  return guard([&] {
    checked(s);
    s->fene.on = 1;
    s->fene.K = K;
    s->fene.r0 = r0;
    s->fene.rmax = rmax;
    s->fene.rmaxsq = rmax * rmax;
    s->fene.rcsq = rc * rc;
    s->fene.shift = shift;
  });
}

int espp_triples_add(espp_system* s, int64_t n, const int64_t* triples) {
  return guard([&] {
    checked(s);
    if (n > 0 && !triples) raise(ESPP_EINVAL, "null triple array");
    std::unordered_map<int64_t, int> have;
    for (int64_t id : s->allIds) have[id] = 1;
    for (int64_t t = 0; t < n; ++t) {
      std::array<int64_t, 3> tr = {triples[3 * t], triples[3 * t + 1], triples[3 * t + 2]};
      for (int64_t id : tr)
        if (!have.count(id)) raise(ESPP_EINVAL, "triple member does not exist");
      s->triples.push_back(tr);
    }
    s->idDirty = true;
  });
}

// FixedTripleList::remove (FixedTripleList.py:97-100): the list is emptied.
int espp_triples_clear(espp_system* s) {
  return guard([&] {
    checked(s)->triples.clear();
    s->idDirty = true;
  });
}

int espp_triples_size(espp_system* s, int64_t* n) {
  return guard([&] { *n = (int64_t)checked(s)->triples.size(); });
}

int espp_cosine_set(espp_system* s, double K, double theta0) {
  return guard([&] {
    checked(s);
    s->cosine.on = 1;
    s->cosine.K = K;
    s->cosine.theta0 = theta0;
    s->cosine.Kcos_theta0 = K * std::cos(theta0);
    s->cosine.Ksin_theta0 = K * std::sin(theta0);
  });
}

int espp_tab_read(const char* path, int64_t cap, double* r, double* energy, double* force,
                  int64_t* n) {
  return guard([&] {
    if (!path || !n) raise(ESPP_EINVAL, "null argument");
    // InterpolationLinear::readFile: fgets + sscanf("%lg %lg %lg"), other lines skipped
    FILE* fp = std::fopen(path, "r");
    if (!fp) raise(ESPP_EINVAL, std::string("could not open file ") + path);
    char line[1024];
    int64_t cnt = 0;
    while (std::fgets(line, sizeof(line), fp)) {
      double a, b, c;
      if (std::sscanf(line, "%lg %lg %lg", &a, &b, &c) < 3) continue;
      if (cnt < cap) {
        if (r) r[cnt] = a;
        if (energy) energy[cnt] = b;
        if (force) force[cnt] = c;
      }
      ++cnt;
    }
    std::fclose(fp);
    *n = cnt;
    if (cnt < 2) raise(ESPP_EINVAL, "illegal file for tabulated potential");
  });
}

int espp_tab_eval(int32_t itype, int64_t n, const double* r, const double* e, const double* f,
                  int64_t m, const double* x, double* energy, double* force) {
  return guard([&] {
    if (!r || !e || !f || (m > 0 && !x)) raise(ESPP_EINVAL, "null argument");
    if (n > 0x7fffffff) raise(ESPP_ERANGE, "table too long");
    TabDesc t;
    std::vector<double> coef;
    if (const char* msg = build_table(itype, (int)n, r, e, f, t, coef)) raise(ESPP_EINVAL, msg);
    for (int64_t k = 0; k < m; ++k) {
      if (energy) energy[k] = tab_value(t, coef.data(), false, x[k]);
      if (force) force[k] = tab_value(t, coef.data(), true, x[k]);
    }
  });
}

namespace {
void set_tab(espp_system* s, int key, int32_t itype, int64_t n, const double* r,
             const double* e, const double* f, double rc, double shift) {
  if (!r || !e || !f) raise(ESPP_EINVAL, "null table");
  if (n > 0x7fffffff) raise(ESPP_ERANGE, "table too long");
  espp_system::TabSpec t;
  t.itype = itype;
  t.r.assign(r, r + n);
  t.e.assign(e, e + n);
  t.f.assign(f, f + n);
  t.rc = rc;
  t.shift = shift;
  TabDesc probe;
  std::vector<double> coef;
  if (const char* msg = build_table(itype, (int)n, r, e, f, probe, coef)) raise(ESPP_EINVAL, msg);
  s->tabSpecs[key] = std::move(t);
  upload_tabs(s);
}
}  // namespace

int espp_tab_pair_set(espp_system* s, int32_t t1, int32_t t2, int32_t itype, int64_t n,
                      const double* r, const double* e, const double* f, double rc,
                      double shift) {
  return guard([&] {
    checked(s);
    if (t1 < 0 || t2 < 0 || t1 >= kMaxTypes || t2 >= kMaxTypes)
      raise(ESPP_ERANGE, "particle type out of range");
    if (t1 > t2) std::swap(t1, t2);
    set_tab(s, t1 * kMaxTypes + t2, itype, n, r, e, f, rc, shift);
  });
}

int espp_tab_bond_set(espp_system* s, int32_t itype, int64_t n, const double* r,
                      const double* e, const double* f, double rc, double shift) {
  return guard([&] {
    checked(s);
    set_tab(s, kTabBondKey, itype, n, r, e, f, rc, shift);
  });
}

int espp_tab_angle_set(espp_system* s, int32_t itype, int64_t n, const double* theta,
                       const double* e, const double* f) {
  return guard([&] {
    checked(s);
    set_tab(s, kTabAngleKey, itype, n, theta, e, f, INFINITY, 0.0);
  });
}

// FixedPairList::getLongtimeMaxBondSqr / resetLongtimeMaxBondSqr (FixedPairList.cpp:82-86):
// the force kernels raise the counter to the longest bond of each force pass.
int espp_bonds_max_sqr(espp_system* s, double* m) {
  return guard([&] {
    checked(s);
    const unsigned long long b = get_counters(s).ltMaxBondSq;
    std::memcpy(m, &b, sizeof(double));
  });
}

int espp_bonds_reset_max(espp_system* s) {
  return guard([&] {
    checked(s);
    DevCounters c = get_counters(s);
    c.ltMaxBondSq = 0ull;
    set_counters(s, c);
    sync(s);
  });
}

int espp_integrator_set(espp_system* s, double dt) {
  return guard([&] {
    checked(s);
    if (dt == 0.0) raise(ESPP_EINVAL, "Timestep 'dt' must be non-zero!");
    s->dt = dt;
  });
}

int espp_step_get(espp_system* s, int64_t* step) {
  return guard([&] { *step = checked(s)->step; });
}

int espp_step_set(espp_system* s, int64_t step) {
  return guard([&] { checked(s)->step = step; });
}

int espp_langevin_set(espp_system* s, int32_t enabled, double gamma, double T, int64_t nexcl,
                      const int64_t* excl) {
  return guard([&] {
    checked(s);
    s->lang_on = enabled != 0;
    s->gamma = gamma;
    s->temperature = T;
    s->langExclIds.assign(excl, excl + nexcl);
    if (s->idDirty || !s->langExcl) {
      s->idDirty = true;
      return;
    }
    // the id map is current: only the thermostat's exclusion flags change, so the
    // particles keep their order and the Verlet list stays valid (setting up a thermostat
    // triggers no re-sort or list build in the reference either)
    std::vector<uint8_t> le(s->idSpan, 0);
    for (int64_t id : s->langExclIds)
      if (id >= s->idMin && id - s->idMin < s->idSpan) le[id - s->idMin] = 1;
    cuda_check(cudaMemcpyAsync(s->langExcl, le.data(), le.size(), cudaMemcpyHostToDevice, s->st),
               "upload");
    sync(s);
  });
}

int espp_capforce_set(espp_system* s, int32_t mode, const double cap[3]) {
  return guard([&] {
    checked(s);
    if (mode < 0 || mode > 2) raise(ESPP_EINVAL, "unknown force-capping mode");
    s->capMode = mode;
    for (int k = 0; k < 3; ++k) s->cap3[k] = cap ? cap[k] : 0.0;
  });
}

int espp_run(espp_system* s, int64_t nsteps) {
  return guard([&] {
    checked(s);
    if (nsteps < 0) raise(ESPP_EINVAL, "negative step count");
    run(s, nsteps);
  });
}

// ---- spatial decomposition: one system per domain --------------------------------------
// The host loop of a decomposition over several domains (DomainDecomposition.cpp:1031-1158
// migration, :1243-1391 ghost frames) moves particles between the domains' systems at a
// re-sort and refreshes the halo copies every step; the phases below split the step loop
// at those points.  The host takes the maximum displacement over the domains and decides
// the re-sort with the device rule (maxDist += sqrt(max |dx|^2) > skin / 2).

namespace {

// sqrt of the integrate1 maximum |dx|^2 since the last call, which is reset
double take_max_disp(espp_system* s) {
  DevCounters c = get_counters(s);
  double m;
  std::memcpy(&m, &c.maxSq, sizeof(double));
  c.maxSq = 0ull;
  set_counters(s, c);
  return std::sqrt(m);
}

}  // namespace

int espp_dd_load(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                 const double* mass, const double* pos, const double* vel, const int32_t* img,
                 const uint8_t* halo) {
  return guard([&] {
    checked(s);
    if (n < 0 || (n > 0 && (!id || !pos))) raise(ESPP_EINVAL, "bad particle arrays");
    if ((int64_t)n > (1LL << 30)) raise(ESPP_ERANGE, "too many particles");
    HostParticles h;
    h.id.assign(id, id + n);
    std::unordered_map<int64_t, int> seen;
    seen.reserve(n);
    std::vector<int64_t> haloIds;
    for (int64_t i = 0; i < n; ++i) {
      if (seen.count(id[i])) raise(ESPP_EINVAL, "duplicate particle id " + std::to_string(id[i]));
      seen[id[i]] = 1;
      const int ty = type ? type[i] : 0;
      if (ty < 0 || ty >= kMaxTypes) raise(ESPP_ERANGE, "particle type out of range [0, 8)");
      h.type.push_back(ty);
      s->maxType = std::max(s->maxType, ty);
      h.mass.push_back(mass ? mass[i] : 1.0);
      for (int k = 0; k < 3; ++k) {
        h.x.push_back(pos[3 * i + k]);  // as integrated: the next step re-sorts and folds
        h.v.push_back(vel ? vel[3 * i + k] : 0.0);
        h.f.push_back(0.0);
        h.img.push_back(img ? img[3 * i + k] : 0);
      }
      if (halo && halo[i]) haloIds.push_back(id[i]);
    }
    upload(s, h);
    upload_lj(s);
    s->allIds = h.id;
    s->haloIds.swap(haloIds);
    s->idDirty = true;
    s->resortFlag = true;
    s->binned = false;
    s->listValid = false;
  });
}

int espp_dd_set_halo_positions(espp_system* s, int64_t n, const int64_t* ids,
                               const double* pos) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids || !pos) raise(ESPP_EINVAL, "null id or position array");
    ensure_id_map(s);
    ensure_stage(s, n);
    cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                               s->st), "upload ids");
    cuda_check(cudaMemcpyAsync(s->stPos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice,
                               s->st), "upload");
    launch_set_by_id(s->view(), (int)n, s->stIds, s->stPos, nullptr, nullptr, s->st);
    unsigned e = read_err(s);
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
    // the pair list stays: halo copies move like the particles they copy
  });
}

int espp_memory_space(int32_t* kind) {
  return guard([&] {
    if (!kind) raise(ESPP_EINVAL, "null output pointer");
    *kind = 1;  // device memory of the system's GPU
  });
}

// Halo refresh without host copies: ids and pos are device arrays of the system's GPU.
int espp_dd_read_positions(espp_system* s, int64_t n, const int64_t* ids, double* pos) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids || !pos) raise(ESPP_EINVAL, "null id or position array");
    if (n > (1LL << 30)) raise(ESPP_ERANGE, "too many ids");
    ensure_id_map(s);
    launch_get_by_id(s->view(), (int)n, ids, pos, nullptr, nullptr, nullptr, s->st);
    unsigned e = read_err(s);  // synchronises the stream: pos is complete on return
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
  });
}

int espp_dd_write_halo(espp_system* s, int64_t n, const int64_t* ids, const double* pos) {
  return guard([&] {
    checked(s);
    if (n <= 0) return;
    if (!ids || !pos) raise(ESPP_EINVAL, "null id or position array");
    if (n > (1LL << 30)) raise(ESPP_ERANGE, "too many ids");
    ensure_id_map(s);
    launch_set_by_id(s->view(), (int)n, ids, pos, nullptr, nullptr, s->st);
    unsigned e = read_err(s);
    if (e & kErrIdRange) {
      cuda_check(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->st), "memset");
      raise(ESPP_EINVAL, "unknown particle id");
    }
  });
}

int espp_dd_run_begin(espp_system* s, int64_t nsteps, double* maxd) {
  return guard([&] {
    checked(s);
    if (nsteps < 0 || !maxd) raise(ESPP_EINVAL, "bad arguments");
    if (!s->haloIds.empty() && (!s->triples.empty() || s->mlp))
      raise(ESPP_EINVAL, "angles and the learned potential are not available with halo "
                         "particles (spatial decomposition)");
    s->ddT0 = now_s();
    s->ddTResort = 0.0;
    s->ddArgs = run_prologue(s, nsteps, s->ddTResort);
    s->ddRun = true;
    s->ddSteps = nsteps;
    s->ddDone = 0;
    *maxd = nsteps > 0 ? take_max_disp(s) : 0.0;
  });
}

int espp_dd_step(espp_system* s, int32_t resort, double* maxd) {
  return guard([&] {
    checked(s);
    if (!maxd) raise(ESPP_EINVAL, "null output pointer");
    if (!s->ddRun || s->ddDone >= s->ddSteps)
      raise(ESPP_ESTATE, "no step of a decomposed run is pending");
    if (resort || s->resortFlag) {
      const double tr = now_s();
      if (s->idDirty) rebuild_id_tables(s);
      timed_decompose(s);
      s->resortFlag = false;
      s->nResorts++;
      s->ddTResort += now_s() - tr;
    }
    timed_forces(s);
    const bool last = s->ddDone + 1 == s->ddSteps;
    IntegrateArgs aj = s->ddArgs;
    aj.step = s->step;
    aj.do_i1 = last ? 0 : 1;
    aj.storeFtot = last ? 1 : 0;
    timed_integrate(s, aj);
    cuda_check(cudaGetLastError(), "step kernels");
    s->step++;
    s->ddDone++;
    *maxd = last ? 0.0 : take_max_disp(s);
  });
}

int espp_dd_run_end(espp_system* s) {
  return guard([&] {
    checked(s);
    if (!s->ddRun) raise(ESPP_ESTATE, "no decomposed run in progress");
    s->ddRun = false;
    cuda_check(cudaEventRecord(s->runEnd, s->st), "event");
    run_epilogue(s, s->ddT0, s->ddTResort, false);
  });
}

int espp_num_resorts(espp_system* s, int64_t* n) {
  return guard([&] { *n = checked(s)->nResorts; });
}

int espp_timers(espp_system* s, double t[10]) {
  return guard([&] {
    checked(s);
    for (int k = 0; k < 10; ++k) t[k] = s->timers[k];
  });
}

int espp_energy(espp_system* s, int32_t which, double* e) {
  return guard([&] {
    double o[7];
    observable(checked(s), which, 1, o);
    *e = o[0];
  });
}

int espp_virial(espp_system* s, int32_t which, double* w) {
  return guard([&] {
    double o[7];
    observable(checked(s), which, 0, o);
    *w = o[0];
  });
}

int espp_virial_tensor(espp_system* s, int32_t which, double w[6]) {
  return guard([&] {
    double o[7];
    observable(checked(s), which, 0, o);
    for (int k = 0; k < 6; ++k) w[k] = o[k + 1];
  });
}

int espp_kinetic(espp_system* s, double* sum_mv2, int64_t* n) {
  return guard([&] {
    checked(s);
    *sum_mv2 = 0.0;
    *n = s->n - (int64_t)s->haloIds.size();
    if (s->n == 0) return;
    int nb;
    double* part = obs_partials(s, nb);
    launch_kinetic(s->view(), part, nb, s->obs, s->st);
    cuda_check(cudaMemcpyAsync(sum_mv2, s->obs, sizeof(double), cudaMemcpyDeviceToHost, s->st),
               "download");
    sync(s);
  });
}

int espp_kinetic_types(espp_system* s, uint64_t type_mask, double* sum_mv2, int64_t* n) {
  return guard([&] {
    checked(s);
    if (!sum_mv2 || !n) raise(ESPP_EINVAL, "null output pointer");
    *sum_mv2 = 0.0;
    *n = 0;
    if (s->n == 0 || type_mask == 0) return;
    int nb;
    double* part = obs_partials(s, nb);
    launch_kinetic_types(s->view(), (unsigned long long)type_mask, part, nb, s->obs, s->st);
    double out[2];
    cuda_check(cudaMemcpyAsync(out, s->obs, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st),
               "download");
    sync(s);
    *sum_mv2 = out[0];
    *n = (int64_t)out[1];
  });
}

int espp_kinetic_tensor(espp_system* s, double out[6]) {
  return guard([&] {
    checked(s);
    if (!out) raise(ESPP_EINVAL, "null output pointer");
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    if (s->n == 0) return;
    int nb;
    double* part = obs_partials(s, nb);
    launch_kinetic_tensor(s->view(), part, nb, s->obs, s->st);
    cuda_check(cudaMemcpyAsync(out, s->obs, 6 * sizeof(double), cudaMemcpyDeviceToHost, s->st),
               "download");
    sync(s);
  });
}

int espp_selftest_bounded_wait(espp_system* s, int64_t spins, double* ns) {
  return guard([&] {
    checked(s);
    if (!(spins >= 1 && spins <= (int64_t)1 << 20))
      raise(ESPP_ERANGE, "spins must lie in [1, 2^20]");
    unsigned long long* d_out = dalloc<unsigned long long>(2);
    unsigned long long h[2] = {0, 0};
    launch_wait_selftest(s->err, (long long)spins, d_out, s->st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    dfree(d_out);
    cuda_check(e, "bounded-wait self-test");
    if (ns) *ns = (double)h[0];
    check_err(s);
    if (h[1] == 0) raise(ESPP_ESTATE, "an mbarrier phase completed with no arrival");
  });
}

int espp_force_acc(espp_system* s, int32_t op, int64_t n, const int64_t* ids, double* out) {
  return guard([&] {
    checked(s);
    ensure_id_map(s);
    if (!s->facc || s->faccSpan != s->idSpan) {
      dfree(s->facc);
      s->facc = dalloc<double>(3 * (size_t)std::max(s->idSpan, 1));
      s->faccSpan = s->idSpan;
      op = 0;
      cuda_check(cudaMemsetAsync(s->facc, 0, sizeof(double) * 3 * std::max(s->idSpan, 1),
                                 s->st), "memset");
    }
    if (op == 0) {
      cuda_check(cudaMemsetAsync(s->facc, 0, sizeof(double) * 3 * std::max(s->idSpan, 1),
                                 s->st), "memset");
    } else if (op == 1) {
      launch_force_acc_add(s->view(), s->facc, s->st);
    } else if (op == 2) {
      if (n <= 0) return;
      if (!ids || !out) raise(ESPP_EINVAL, "null argument");
      ensure_stage(s, n);
      cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                                 s->st), "upload");
      launch_force_acc_read(s->view(), (int)n, s->stIds, s->facc, s->stF, s->st);
      cuda_check(cudaMemcpyAsync(out, s->stF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                                 s->st), "download");
      sync(s);
      check_err(s);
    } else {
      raise(ESPP_EINVAL, "op must be 0 (clear), 1 (add) or 2 (read)");
    }
    cuda_check(cudaGetLastError(), "force accumulator");
  });
}

int espp_mlp_create(double rc, double r0, espp_mlp** out) {
  return guard([&] {
    if (!out) raise(ESPP_EINVAL, "null output pointer");
    if (!(rc > r0) || r0 < 0) raise(ESPP_EINVAL, "the basis needs 0 <= r0 < rc");
    auto m = std::make_unique<espp_mlp>();
    cuda_check(cudaGetDevice(&m->device), "cudaGetDevice");
    m->rc = rc;
    m->r0 = r0;
    if (const char* e = std::getenv("ESPP_B200_MLP_TC")) m->tensor_cores = std::atoi(e) ? 1 : 0;
    m->theta = dalloc<float>(kMlpParams);
    m->grad = dalloc<float>(kMlpParams);
    m->adam_m = dalloc<float>(kMlpParams);
    m->adam_v = dalloc<float>(kMlpParams);
    m->shift = dalloc<float>(kMlpK);
    m->scale = dalloc<float>(kMlpK);
    for (float* p : {m->theta, m->grad, m->adam_m, m->adam_v})
      cuda_check(cudaMemset(p, 0, sizeof(float) * kMlpParams), "memset");
    std::vector<float> zero(kMlpK, 0.f), one(kMlpK, 1.f);
    cuda_check(cudaMemcpy(m->shift, zero.data(), sizeof(float) * kMlpK, cudaMemcpyHostToDevice),
               "upload");
    cuda_check(cudaMemcpy(m->scale, one.data(), sizeof(float) * kMlpK, cudaMemcpyHostToDevice),
               "upload");
    *out = m.release();
  });
}

int espp_mlp_set_mode(espp_mlp* m, int32_t tensor_cores) {
  return guard([&] {
    if (!m) raise(ESPP_EINVAL, "null model");
    m->tensor_cores = tensor_cores ? 1 : 0;
  });
}

int espp_mlp_destroy(espp_mlp* m) {
  return guard([&] {
    if (!m) return;
    cudaSetDevice(m->device);
    for (float* p : {m->theta, m->grad, m->adam_m, m->adam_v, m->shift, m->scale})
      if (p) cudaFree(p);
    delete m;
  });
}

int espp_mlp_num_params(int64_t* n) {
  return guard([&] {
    if (!n) raise(ESPP_EINVAL, "null output pointer");
    *n = kMlpParams;
  });
}

int espp_mlp_set_params(espp_mlp* m, int64_t n, const double* theta) {
  return guard([&] {
    if (!m || !theta) raise(ESPP_EINVAL, "null argument");
    if (n != kMlpParams) raise(ESPP_EINVAL, "wrong number of parameters");
    cuda_check(cudaSetDevice(m->device), "cudaSetDevice");
    std::vector<float> h(theta, theta + n);
    cuda_check(cudaMemcpy(m->theta, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice),
               "upload");
  });
}

int espp_mlp_get_params(espp_mlp* m, int64_t n, double* theta) {
  return guard([&] {
    if (!m || !theta) raise(ESPP_EINVAL, "null argument");
    if (n != kMlpParams) raise(ESPP_EINVAL, "wrong number of parameters");
    cuda_check(cudaSetDevice(m->device), "cudaSetDevice");
    std::vector<float> h(n);
    cuda_check(cudaMemcpy(h.data(), m->theta, sizeof(float) * n, cudaMemcpyDeviceToHost),
               "download");
    for (int64_t q = 0; q < n; ++q) theta[q] = h[q];
  });
}

int espp_mlp_set_norm(espp_mlp* m, const double* shift, const double* scale) {
  return guard([&] {
    if (!m || !shift || !scale) raise(ESPP_EINVAL, "null argument");
    cuda_check(cudaSetDevice(m->device), "cudaSetDevice");
    std::vector<float> a(shift, shift + kMlpK), b(scale, scale + kMlpK);
    cuda_check(cudaMemcpy(m->shift, a.data(), sizeof(float) * kMlpK, cudaMemcpyHostToDevice),
               "upload");
    cuda_check(cudaMemcpy(m->scale, b.data(), sizeof(float) * kMlpK, cudaMemcpyHostToDevice),
               "upload");
  });
}

int espp_mlp_attach(espp_system* s, espp_mlp* m) {
  return guard([&] {
    checked(s);
    if (m && m->device != s->device) raise(ESPP_EINVAL, "model and system on different devices");
    if (m && s->has_vl && s->vl_cut < m->rc)
      raise(ESPP_ERANGE, "Verlet-list cutoff below the model's cutoff");
    s->mlp = m;
    s->mlpCap = 0;
    ensure_mlp_scratch(s);
  });
}

int espp_mlp_descriptors(espp_system* s, int64_t n, const int64_t* ids, double* G) {
  return guard([&] {
    checked(s);
    if (!s->mlp || !s->has_vl) raise(ESPP_ESTATE, "no learned potential on a Verlet list");
    prepare_observables(s);
    DevView d = s->view();
    launch_mlp_energy_terms(d, s->st);
    sync_pa(s);
    std::vector<float> g((size_t)s->n * kMlpK);
    std::vector<int64_t> sid(s->n);
    cuda_check(cudaMemcpyAsync(g.data(), s->mlpG, sizeof(float) * g.size(),
                               cudaMemcpyDeviceToHost, s->st), "download");
    cuda_check(cudaMemcpyAsync(sid.data(), s->A.id, sizeof(int64_t) * s->n,
                               cudaMemcpyDeviceToHost, s->st), "download");
    sync(s);
    std::unordered_map<int64_t, int> where;
    where.reserve(s->n * 2);
    for (int i = 0; i < s->n; ++i) where[sid[i]] = i;
    for (int64_t k = 0; k < n; ++k) {
      auto it = where.find(ids[k]);
      if (it == where.end()) raise(ESPP_EINVAL, "particle id not present");
      for (int q = 0; q < kMlpK; ++q) G[k * kMlpK + q] = g[(size_t)it->second * kMlpK + q];
    }
  });
}

int espp_mlp_fm_grad(espp_system* s, int64_t n, const int64_t* ids, const double* fref,
                     double* loss, double* grad) {
  return guard([&] {
    checked(s);
    if (!s->mlp || !s->has_vl) raise(ESPP_ESTATE, "no learned potential on a Verlet list");
    if (n != s->n) raise(ESPP_EINVAL, "reference forces must cover every particle");
    prepare_observables(s);
    ensure_stage(s, n);
    DevView d = s->view();
    cuda_check(cudaMemcpyAsync(s->stIds, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s->st),
               "upload");
    cuda_check(cudaMemcpyAsync(s->stPos, fref, sizeof(double) * 3 * n, cudaMemcpyHostToDevice,
                               s->st), "upload");
    launch_scatter3_by_id(d, (int)n, s->stIds, s->stPos, s->mlpFref, s->st);
    std::vector<float> g0;
    if (grad) {
      g0.resize(kMlpParams);
      cuda_check(cudaMemcpyAsync(g0.data(), s->mlp->grad, sizeof(float) * kMlpParams,
                                 cudaMemcpyDeviceToHost, s->st), "download");
    }
    launch_mlp_forces(d, false, s->mlpF, s->st);
    int nb;
    double* part = obs_partials(s, nb);
    launch_mlp_fm_grad(d, s->mlpF, s->mlpFref, s->mlpErr, s->mlpTan, s->mlpPart,
                       mlp_grad_blocks(s->n), s->mlp->grad, part, nb, s->obs, s->st);
    cuda_check(cudaGetLastError(), "force-matching kernels");
    double l = 0.0;
    cuda_check(cudaMemcpyAsync(&l, s->obs, sizeof(double), cudaMemcpyDeviceToHost, s->st),
               "download");
    std::vector<float> g1;
    if (grad) {
      g1.resize(kMlpParams);
      cuda_check(cudaMemcpyAsync(g1.data(), s->mlp->grad, sizeof(float) * kMlpParams,
                                 cudaMemcpyDeviceToHost, s->st), "download");
    }
    sync(s);
    check_err(s);
    if (loss) *loss = l;
    if (grad)
      for (int q = 0; q < kMlpParams; ++q) grad[q] = (double)g1[q] - (double)g0[q];
  });
}

int espp_mlp_adam_step(espp_mlp* m, double lr, double beta1, double beta2, double eps,
                       double gscale) {
  return guard([&] {
    if (!m) raise(ESPP_EINVAL, "null model");
    cuda_check(cudaSetDevice(m->device), "cudaSetDevice");
    launch_mlp_adam(m, lr, beta1, beta2, eps, gscale, 0);
    cuda_check(cudaGetLastError(), "adam kernel");
    cuda_check(cudaDeviceSynchronize(), "adam");
  });
}

int espp_rdf(espp_system* s, int32_t rdfN, double* out) {
  return guard([&] {
    checked(s);
    if (rdfN <= 0 || !out) raise(ESPP_EINVAL, "rdfN must be positive");
    if (!s->haloIds.empty())
      raise(ESPP_EINVAL, "the RDF is not available with halo particles (spatial decomposition)");
    if (s->idDirty) rebuild_id_tables(s);
    if (!s->binned) bin(s, false);
    // dr from half the y edge, as the reference does (RadialDistrF.cpp:59-60)
    const double dr = (s->L[1] / 2.) / (double)rdfN;
    unsigned long long* hist = dalloc<unsigned long long>(rdfN);
    std::vector<unsigned long long> h(rdfN);
    try {
      cuda_check(cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * rdfN, s->st), "memset");
      launch_rdf(s->view(), rdfN, dr, hist, s->st);
      cuda_check(cudaGetLastError(), "rdf kernel");
      cuda_check(cudaMemcpyAsync(h.data(), hist, sizeof(unsigned long long) * rdfN,
                                 cudaMemcpyDeviceToHost, s->st), "download");
      sync(s);
    } catch (...) {
      dfree(hist);
      throw;
    }
    dfree(hist);
    // normalisation (RadialDistrF.cpp:136-146): the factor is formed in long double
    const int num_part = s->n;
    const double rho = (double)num_part / (s->L[0] * s->L[1] * s->L[2]);
    const double factor = 2.0 * 3.141592653589793238462643383279502884L * dr * rho *
                          (double)1 * (double)num_part;
    for (int i = 0; i < rdfN; i++) {
      const double radius = (i + 0.5) * dr;
      out[i] = (double)h[i] / (factor * (radius * radius + dr * dr / 12.0));
    }
  });
}

// ---- snapshots of tracked particles, mean-square displacement ----------------------

struct espp_confs {
  espp_system* s = nullptr;
  int key = 0;
  int64_t n = 0;
  int64_t* ids = nullptr;    // device, tracked ids in order
  double* snap = nullptr;    // device, M snapshots of 3 n doubles
  int M = 0, capM = 0;
};

namespace espp {
namespace {
void confs_reserve(espp_confs* c, int M) {
  if (M <= c->capM) return;
  const int cap = std::max(M, std::max(8, 2 * c->capM));
  double* nb = dalloc<double>((size_t)cap * 3 * std::max<int64_t>(c->n, 1));
  if (c->M > 0)
    cuda_check(cudaMemcpyAsync(nb, c->snap, sizeof(double) * 3 * (size_t)c->n * c->M,
                               cudaMemcpyDeviceToDevice, c->s->st), "copy");
  sync(c->s);
  dfree(c->snap);
  c->snap = nb;
  c->capM = cap;
}
// per-lag sums from the per-block partials, in block order
void msd_finish(espp_confs* c, int64_t n, const double* dsnap, double* Z) {
  const int M = c->M;
  const int nb = msd_blocks(n);
  double* part = dalloc<double>((size_t)M * nb);
  std::vector<double> h((size_t)M * nb);
  try {
    launch_msd(dsnap, n, M, part, c->s->st);
    cuda_check(cudaGetLastError(), "msd kernel");
    cuda_check(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                               c->s->st), "download");
    sync(c->s);
  } catch (...) {
    dfree(part);
    throw;
  }
  dfree(part);
  for (int m = 0; m < M; ++m) {
    double z = 0.0;
    for (int b = 0; b < nb; ++b) z += h[(size_t)m * nb + b];
    Z[m] = z;
  }
}
}  // namespace
}  // namespace espp

int espp_confs_create(espp_system* s, int32_t key, int64_t n, const int64_t* ids,
                      espp_confs** out) {
  return guard([&] {
    checked(s);
    if (!out) raise(ESPP_EINVAL, "null output pointer");
    if (key < ESPP_CONF_POSITION || key > ESPP_CONF_UNFOLDED)
      raise(ESPP_EINVAL, "Error. Key is unknown. Use position, unfolded or velocity.");
    if (n < 0 || (n > 0 && !ids)) raise(ESPP_EINVAL, "bad id list");
    auto c = std::make_unique<espp_confs>();
    c->s = s;
    c->key = key;
    c->n = n;
    if (n > 0) {
      c->ids = dalloc<int64_t>((size_t)n);
      cuda_check(cudaMemcpyAsync(c->ids, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s->st),
                 "upload");
      sync(s);
    }
    *out = c.release();
  });
}

int espp_confs_destroy(espp_confs* c) {
  return guard([&] {
    if (!c) return;
    dfree(c->ids);
    dfree(c->snap);
    delete c;
  });
}

int espp_confs_gather(espp_confs* c) {
  return guard([&] {
    if (!c) raise(ESPP_EINVAL, "null handle");
    espp_system* s = c->s;
    checked(s);
    ensure_id_map(s);
    confs_reserve(c, c->M + 1);
    launch_conf_gather(s->view(), c->ids, c->n, c->key, c->snap + (size_t)c->M * 3 * c->n, s->st);
    cuda_check(cudaGetLastError(), "gather kernel");
    sync(s);
    check_err(s);
    ++c->M;
  });
}

int espp_confs_push(espp_confs* c, const double* xyz) {
  return guard([&] {
    if (!c) raise(ESPP_EINVAL, "null handle");
    if (c->n > 0 && !xyz) raise(ESPP_EINVAL, "null argument");
    confs_reserve(c, c->M + 1);
    if (c->n > 0)
      cuda_check(cudaMemcpyAsync(c->snap + (size_t)c->M * 3 * c->n, xyz, sizeof(double) * 3 * c->n,
                                 cudaMemcpyHostToDevice, c->s->st), "upload");
    sync(c->s);
    ++c->M;
  });
}

int espp_confs_size(espp_confs* c, int32_t* m) {
  return guard([&] {
    if (!c || !m) raise(ESPP_EINVAL, "null argument");
    *m = c->M;
  });
}

int espp_confs_clear(espp_confs* c) {
  return guard([&] {
    if (!c) raise(ESPP_EINVAL, "null handle");
    c->M = 0;
  });
}

int espp_confs_get(espp_confs* c, int32_t m, double* xyz) {
  return guard([&] {
    if (!c || !xyz) raise(ESPP_EINVAL, "null argument");
    if (m < 0 || m >= c->M) raise(ESPP_ERANGE, "Error. Velocities::get <out-of-range>");
    if (c->n > 0)
      cuda_check(cudaMemcpyAsync(xyz, c->snap + (size_t)m * 3 * c->n, sizeof(double) * 3 * c->n,
                                 cudaMemcpyDeviceToHost, c->s->st), "download");
    sync(c->s);
  });
}

int espp_msd(espp_confs* c, double* out) {
  return guard([&] {
    if (!c || !out) raise(ESPP_EINVAL, "null argument");
    const int M = c->M;
    if (M == 0) return;
    std::vector<double> Z(M);
    msd_finish(c, c->n, c->snap, Z.data());
    // MeanSquareDispl.cpp:127-137: divide by the number of pairs of snapshots, then by 6 N
    const double inv_coef = 1.0 / (6.0 * (double)c->n);
    for (int m = 0; m < M; ++m) {
      Z[m] /= (double)(M - m);
      out[m] = Z[m] * inv_coef;
    }
  });
}

int espp_msd_chain_com(espp_confs* c, int32_t chainlength, double* out) {
  return guard([&] {
    if (!c || !out) raise(ESPP_EINVAL, "null argument");
    if (chainlength <= 0) raise(ESPP_EINVAL, "chainlength must be positive");
    const int M = c->M;
    const int64_t nch = c->n / chainlength;
    if (M == 0) return;
    if (nch == 0) raise(ESPP_EINVAL, "no complete chain among the tracked particles");
    double* com = dalloc<double>((size_t)M * 3 * nch);
    std::vector<double> Z(M);
    try {
      launch_chain_com(c->snap, c->n, M, chainlength, nch, com, c->s->st);
      cuda_check(cudaGetLastError(), "chain centre kernels");
      // the centres relative to their snapshot mean are the items of the same lag sums
      espp_confs tmp;
      tmp.s = c->s;
      tmp.M = M;
      msd_finish(&tmp, nch, com, Z.data());
    } catch (...) {
      dfree(com);
      throw;
    }
    dfree(com);
    // MeanSquareDispl.cpp:419-425
    const double inv_coef = 1.0 / (6.0 * (double)nch);
    for (int m = 0; m < M; ++m) out[m] = inv_coef * Z[m] / (double)(M - m);
  });
}

int espp_fp32_peak(double* tflops) {
  return guard([&] {
    if (!tflops) raise(ESPP_EINVAL, "null output pointer");
    int dev = 0, nsm = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "attribute");
    *tflops = measure_fp32_tflops(nsm, 0);
    cuda_check(cudaGetLastError(), "fp32 probe");
  });
}

int espp_set_half_cell_int(espp_system* s, int32_t h) {
  return guard([&] {
    checked(s);
    if (h < 1 || h > 4) raise(ESPP_EINVAL, "halfCellInt must be 1 .. 4");
    for (int k = 0; k < 3; ++k)
      if (s->nc[k] < 2 * h + 1)
        raise(ESPP_EINVAL, "the cell grid needs at least 2 halfCellInt + 1 cells a dimension");
    if (s->n > 0) raise(ESPP_ESTATE, "halfCellInt is set before particles are added");
    s->hci = h;
    s->listValid = false;
  });
}

int espp_set_tpp(espp_system* s, int32_t tpp) {
  return guard([&] {
    checked(s);
    if (tpp != 1 && tpp != 2 && tpp != 4 && tpp != 8)
      raise(ESPP_EINVAL, "threads per particle must be 1, 2, 4 or 8");
    s->tpp = tpp;
  });
}

namespace {

// Puts the list into `form` (0: per-particle global list with tpp threads per particle,
// 1: brick windows of extent b, zeros choosing it from the density) at the current
// positions; the rebuild is not counted as a list build.
void apply_layout(espp_system* s, int form, int tpp, const int b[3]) {
  s->brickBuild = form == 2;
  if (form == 1 || form == 2) {
    for (int k = 0; k < 3; ++k) s->brickB[k] = (b && b[k] > 0) ? std::min(b[k], s->nc[k]) : 0;
    if (s->brickB[0] == 0 || s->brickB[1] == 0 || s->brickB[2] == 0)
      s->brickB[0] = s->brickB[1] = s->brickB[2] = 0;
    s->brickWmax = 0;
  }
  if (form == 2) {
    s->brickAllowed = false;
    if (tpp == 1 || tpp == 2 || tpp == 4 || tpp == 8) s->tpp = tpp;
  } else if (form == 1) {
    s->brickAllowed = true;
    for (int k = 0; k < 3; ++k) s->brickB[k] = (b && b[k] > 0) ? std::min(b[k], s->nc[k]) : 0;
    if (s->brickB[0] == 0 || s->brickB[1] == 0 || s->brickB[2] == 0)
      s->brickB[0] = s->brickB[1] = s->brickB[2] = 0;
    s->brickWmax = 0;
  } else {
    s->brickAllowed = false;
    if (tpp == 1 || tpp == 2 || tpp == 4 || tpp == 8) s->tpp = tpp;
  }
  if (s->idDirty) rebuild_id_tables(s);
  if (!s->binned) bin(s, false);
  if (!s->has_vl) return;
  const int64_t builds = s->builds;
  build_list(s);
  s->builds = builds;
}

// Device time (ms) of one list build in the current form and the mean of 3 force
// launches on it.
void time_layout(espp_system* s, double& build_ms, double& force_ms) {
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  const double cv = s->vl_cut + s->skin;
  DevView d = s->view();
  cuda_check(cudaEventRecord(e0, s->st), "event");
  if (s->brickOn || s->brickBuildUsed)
    launch_build_brick(d, cv * cv, s->st);
  else
    launch_build_nl(d, cv * cv, true, s->st);  // the form the step loop's rebuilds use
  cuda_check(cudaEventRecord(e1, s->st), "event");
  sync(s);
  float t = 0.f;
  cuda_check(cudaEventElapsedTime(&t, e0, e1), "event time");
  build_ms = t;
  launch_force_kernel(s, s->st);  // warm
  cuda_check(cudaEventRecord(e0, s->st), "event");
  for (int r = 0; r < 3; ++r) launch_force_kernel(s, s->st);
  cuda_check(cudaEventRecord(e1, s->st), "event");
  sync(s);
  cuda_check(cudaEventElapsedTime(&t, e0, e1), "event time");
  force_ms = t / 3.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cuda_check(cudaGetLastError(), "layout timing");
  check_err(s);
}

}  // namespace

int espp_set_layout(espp_system* s, int32_t form, int32_t tpp, const int32_t brick[3]) {
  return guard([&] {
    checked(s);
    if (form < 0 || form > 2) raise(ESPP_EINVAL, "layout form must be 0, 1 or 2");
    if (form != 1 && tpp != 1 && tpp != 2 && tpp != 4 && tpp != 8)
      raise(ESPP_EINVAL, "threads per particle must be 1, 2, 4 or 8");
    int b[3] = {0, 0, 0};
    for (int k = 0; k < 3 && brick; ++k) {
      if (brick[k] < 0 || brick[k] > kBrickMax)
        raise(ESPP_EINVAL, "brick extent must be 0 (automatic) or 1.." + std::to_string(kBrickMax));
      b[k] = brick[k];
    }
    apply_layout(s, form, tpp, b);
  });
}

int espp_get_layout(espp_system* s, int32_t out[5]) {
  return guard([&] {
    checked(s);
    if (!out) raise(ESPP_EINVAL, "null output pointer");
    out[0] = s->brickOn ? 1 : (s->brickBuildUsed ? 2 : 0);
    out[1] = s->tpp;
    for (int k = 0; k < 3; ++k) out[2 + k] = (s->brickOn || s->brickBuildUsed) ? s->brickB[k] : 0;
  });
}

int espp_autotune_layout(espp_system* s, double steps_per_build, int32_t best[5],
                         double* table, int32_t cap, int32_t* ncand) {
  return guard([&] {
    checked(s);
    if (s->idDirty) rebuild_id_tables(s);
    if (!s->binned) bin(s, false);
    if (!s->has_vl) raise(ESPP_ESTATE, "no Verlet list");
    const double interval = steps_per_build > 0 ? steps_per_build : 10.0;
    struct Cand {
      int form, tpp, b[3];
    };
    std::vector<Cand> cands;
    for (int t : {1, 2, 4, 8}) cands.push_back({0, t, {0, 0, 0}});
    if (brick_geometry_ok(s))
      for (int t : {1, 2, 4}) cands.push_back({2, t, {0, 0, 0}});
    const bool brickable = [&] {
      const bool was = s->brickAllowed;
      s->brickAllowed = true;
      const bool ok = brick_wanted(s);
      s->brickAllowed = was;
      return ok;
    }();
    if (brickable) {
      const int shapes[][3] = {{0, 0, 0}, {1, 2, 2}, {2, 2, 2}, {2, 2, 3}, {2, 3, 3},
                               {3, 3, 3}, {4, 4, 4}};
      for (auto& sh : shapes) cands.push_back({1, 0, {sh[0], sh[1], sh[2]}});
    }
    double bestScore = 1e300;
    int pick = -1;
    int row = 0;
    for (size_t c = 0; c < cands.size(); ++c) {
      apply_layout(s, cands[c].form, cands[c].tpp, cands[c].b);
      if (cands[c].form == 1 && !s->brickOn) continue;       // the window did not fit
      if (cands[c].form == 2 && !s->brickBuildUsed) continue;
      double bms = 0.0, fms = 0.0;
      time_layout(s, bms, fms);
      const double score = fms + bms / interval;
      if (table && row < cap) {
        double* r = table + (size_t)row * 8;
        r[0] = cands[c].form;
        r[1] = cands[c].form != 1 ? cands[c].tpp : 0;
        for (int k = 0; k < 3; ++k) r[2 + k] = cands[c].form != 0 ? s->brickB[k] : 0;
        r[5] = fms;
        r[6] = bms;
        r[7] = score;
      }
      ++row;
      if (score < bestScore) {
        bestScore = score;
        pick = (int)c;
      }
    }
    if (pick < 0) raise(ESPP_ESTATE, "no list layout could be timed");
    apply_layout(s, cands[pick].form, cands[pick].tpp, cands[pick].b);
    if (ncand) *ncand = row;
    if (best) {
      best[0] = s->brickOn ? 1 : (s->brickBuildUsed ? 2 : 0);
      best[1] = s->tpp;
      for (int k = 0; k < 3; ++k)
        best[2 + k] = (s->brickOn || s->brickBuildUsed) ? s->brickB[k] : 0;
    }
  });
}

int espp_autotune(espp_system* s, int32_t* best_tpp, double ms[4]) {
  return guard([&] {
    checked(s);
    if (s->idDirty) rebuild_id_tables(s);
    if (!s->binned) bin(s, false);
    if (s->has_vl && !s->listValid) build_list(s);
    const int cand[4] = {1, 2, 4, 8};
    const int old = s->tpp;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    double best = 1e300;
    int pick = old;
    for (int c = 0; c < 4; ++c) {
      s->tpp = cand[c];
      launch_force_kernel(s, s->st);  // warm
      cuda_check(cudaEventRecord(e0, s->st), "event");
      for (int r = 0; r < 3; ++r) launch_force_kernel(s, s->st);
      cuda_check(cudaEventRecord(e1, s->st), "event");
      sync(s);
      float t = 0.f;
      cuda_check(cudaEventElapsedTime(&t, e0, e1), "event time");
      if (ms) ms[c] = t / 3.0;
      if (t < best) {
        best = t;
        pick = cand[c];
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cuda_check(cudaGetLastError(), "autotune");
    check_err(s);
    s->tpp = pick;
    if (best_tpp) *best_tpp = pick;
  });
}

int espp_batch_create(espp_system* const* systems, int32_t n, espp_batch** out) {
  return guard([&] {
    if (!systems || !out || n <= 0) raise(ESPP_EINVAL, "need at least one system");
    std::unique_ptr<espp_batch> b(new espp_batch());
    for (int32_t k = 0; k < n; ++k) {
      if (!systems[k]) raise(ESPP_EINVAL, "null system handle");
      if (k > 0 && systems[k]->device != systems[0]->device)
        raise(ESPP_EINVAL, "all systems of a batch must live on the same device");
      for (int32_t m = 0; m < k; ++m)
        if (systems[m] == systems[k]) raise(ESPP_EINVAL, "a system appears twice in the batch");
      b->sys.push_back(systems[k]);
    }
    b->device = systems[0]->device;
    cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "stream");
    cuda_check(cudaEventCreate(&b->beg), "event");
    cuda_check(cudaEventCreate(&b->end), "event");
    b->ready.resize(n);
    for (auto& e : b->ready) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    *out = b.release();
  });
}

int espp_batch_destroy(espp_batch* b) {
  return guard([&] {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_destroy_graph(b);
    for (auto& e : b->ready) cudaEventDestroy(e);
    if (b->beg) cudaEventDestroy(b->beg);
    if (b->end) cudaEventDestroy(b->end);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
  });
}

int espp_batch_run(espp_batch* b, int64_t nsteps) {
  return guard([&] {
    if (!b) raise(ESPP_EINVAL, "null batch handle");
    if (nsteps < 0) raise(ESPP_EINVAL, "negative step count");
    cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
    for (espp_system* s : b->sys)
      if (s->profiling) raise(ESPP_ESTATE, "profiling is on for a system of the batch");
    batch_run(b, nsteps);
  });
}

int espp_batch_last_run_ms(espp_batch* b, double* ms) {
  return guard([&] {
    if (!b) raise(ESPP_EINVAL, "null batch handle");
    *ms = b->lastMs;
  });
}

int espp_energy_noalloc(espp_system* s, int32_t which, double* e) {
  return guard([&] {
    checked(s);
    if (!e) raise(ESPP_EINVAL, "null output pointer");
    if (which != ESPP_IA_LJ && which != ESPP_IA_FENE)
      raise(ESPP_EINVAL, "unknown interaction kind");
    if (s->n > kNoAllocMaxParticles)
      raise(ESPP_ERANGE, "espp_energy_noalloc handles at most 8388608 particles (its static "
                         "scratch holds 32768 reduction blocks of 256); use espp_energy");
    // everything the reduction reads must already exist: this call builds nothing
    if (s->idDirty || !s->binned || (which == ESPP_IA_LJ && s->has_vl && s->lj_any &&
                                     !s->listValid))
      raise(ESPP_ESTATE, "espp_energy_noalloc needs particles sorted and the Verlet list "
                         "built (call espp_decompose, espp_run or espp_energy first)");
    double* scratch = noalloc_scratch(s->device);
    *e = 0.0;
    if (s->n == 0) return;
    if (which == ESPP_IA_LJ && (!s->has_vl || !s->lj_any)) return;
    if (which == ESPP_IA_FENE && !s->fene.on) return;
    // every slot read below is written first: each block stores its own partial row and
    // the final kernel overwrites the 7 result slots, so nothing needs clearing
    const int nb = observable_blocks(s->n);
    double* partials = scratch + 8;
    double* out = scratch;
    DevView d = s->view();
    if (which == ESPP_IA_LJ && s->brickOn) {
      if (d.brick.nbricks > kNoAllocMaxBlocks)
        raise(ESPP_ERANGE, "espp_energy_noalloc handles at most 32768 bricks; use espp_energy");
      launch_lj_observables_brick(d, partials, 0, out, 1, s->st);
    } else if (which == ESPP_IA_LJ) {
      launch_lj_observables(d, partials, nb, out, 1, s->st);
    } else
      launch_fene_observables(d, s->fene, partials, nb, out, 1, s->st);
    cuda_check(cudaGetLastError(), "energy kernels");
    cuda_check(cudaMemcpyAsync(e, out, sizeof(double), cudaMemcpyDeviceToHost, s->st),
               "download");
    sync(s);
  });
}

}  // extern "C"
