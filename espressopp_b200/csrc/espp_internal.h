// espp_internal.h - device data layout and kernel launch interface shared by the host
// runtime (espp_api.cu) and the kernels (espp_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace espp {

constexpr int kMaxTypes = 8;
constexpr double kFix = 4294967296.0;        // 2^32: fixed-point force scale
constexpr double kInvFix = 1.0 / 4294967296.0;

#ifdef __CUDACC__
// Verlet list layout: each particle's entries in blocks of 8 contiguous ints, block b of
// particle i at ints [(b * cap + i) * 8, +8).  A thread reads a whole block with two
// 16-byte loads and a warp of consecutive particles reads 1 KB of contiguous memory.
__host__ __device__ __forceinline__ size_t nl_index(int k, int i, size_t cap) {
  return (((size_t)(k >> 3) * cap + (size_t)i) << 3) + (size_t)(k & 7);
}
#endif

// device error word bits
enum : unsigned {
  kErrNlOverflow = 1u << 0,    // a particle has more Verlet neighbours than the capacity
  kErrFixOverflow = 1u << 1,   // |F| beyond the int64 2^-32 fixed-point range
  kErrOutside = 1u << 2,       // non-finite or out-of-grid coordinate at re-binning
  kErrBondMissing = 1u << 3,   // bond partner id not present
  kErrIdRange = 1u << 4,       // particle id outside the dense id map
  kErrTimeout = 1u << 5,       // a bounded wait inside a kernel ran out
  kErrWindow = 1u << 6,        // a brick window holds more particles than its stage
};

// Lennard-Jones parameters of one type pair (LennardJones.hpp:79-87 preset()).
struct LJPair {
  double ff1, ff2;   // 48 eps sig^12, 24 eps sig^6
  double ef1, ef2;   // 4 eps, sig^2 (energy uses 4 eps ((sig^2/r^2)^6 - (sig^2/r^2)^3))
  double rcsq;       // cutoff^2 (pairs with r^2 > rcsq feel nothing)
  double shift;      // energy shift
  double caprad;     // > 0: LennardJonesCapped
  double capff;      // capped branch: 48 eps frac6 (frac6 - 0.5) / caprad
  int set;
  int pad;
};

struct LJTable {
  int ntypes;
  int single;        // one type pair only: skip the type lookup
  LJPair p[kMaxTypes * kMaxTypes];
};

// float copy of the table used by the mixed-precision force kernel
struct LJPairF {
  float ff1, ff2, rcsq, capsq, capff;
  int set;
};

struct FENEParams {
  int on;
  double K, r0, rmax, rmaxsq, rcsq, shift;
};

// interaction::Cosine on a FixedTripleList (src/interaction/Cosine.hpp:38-125):
// E = K (1 + cos(theta - theta0)).
struct CosineParams {
  int on;
  double K, theta0, Kcos_theta0, Ksin_theta0;
};

// Per-particle arrays in cell-sorted order.  Two copies exist; the re-sort gathers
// from one into the other and swaps.
struct ParticleArrays {
  double* x;     // 3*cap, SoA: x[0..cap) y[cap..2cap) z[2cap..3cap)
  double* v;     // 3*cap
  int64_t* id;   // cap
  int32_t* type; // cap
  double* mass;  // cap
  int32_t* img;  // 3*cap
};

// Step-loop state kept on the device so that a captured CUDA graph can run the loop.
struct DevCounters {
  unsigned long long maxSq;  // max |dx|^2 of the last integrate1, as double bits
  double maxDist;            // accumulated max displacement since the last re-sort
  long long step;            // step whose force is being computed (Langevin counter)
  long long remaining;       // loop steps left after the current one
  long long resorts;         // re-sorts done in this run
  int flag;                  // re-sort needed this step
  int nnMax;                 // largest neighbour count seen by the Verlet builds
  double pref1, pref2;       // Langevin prefactors of the step loop (-gamma, sqrt(24 T gamma/dt))
  unsigned long long ltMaxBondSq;  // longest bond^2 seen by the force passes, as double bits
};

// Pointers and scalars every kernel needs; passed by value.
// Learned coarse-grained pair potential (per-site radial-basis descriptor -> MLP ->
// site energy), device view.  K = 16 basis functions, H = 64 hidden units.
constexpr int kMlpK = 16;
constexpr int kMlpH = 64;
constexpr int kMlpParams = kMlpH * kMlpK + kMlpH + kMlpH * kMlpH + kMlpH + kMlpH + 1;
struct MlpDev {
  float rc, gamma;        // g_k(r) = exp(-gamma (r - mu_k)^2) fc(r), fc = (cos(pi r/rc) + 1)/2
  float r0, dmu;          // mu_k = r0 + k dmu
  const float* theta;     // W1[H][K], b1[H], W2[H][H], b2[H], w3[H], b3
  const float* shift;     // K: x = (G - shift) * scale feeds the network
  const float* scale;
  float* G;               // per particle: descriptor (cap x K)
  float* D;               // per particle: dE/dG (cap x K)
  float* E;               // per particle: site energy (cap)
  int on;
  int tc;                 // site network on the tensor cores (BF16) instead of FP32
};

// One interpolation table of interaction::Tabulated (InterpolationLinear / Akima / Cubic)
// with the potential's cutoff and shift.  Coefficients live in one double array:
// r[n] at off_r; energy and force coefficient arrays at off_e / off_f, laid out per
// interpolation type: linear a[n], b[n]; Akima p0[n], p1[n], p2[n], p3[n]; cubic y[n],
// y2[n] (value and second derivative of the spline).
struct TabDesc {
  int itype;
  int n;
  int off_r, off_e, off_f;
  double inner, invdelta, deltasq6;
  double rcsq, shift;
};

// Brick path of the Verlet build and the pair kernels: the cell grid tiled into bricks
// of b[0] x b[1] x b[2] cells.  A brick's window (its cells and one layer of cells
// around them) holds every candidate of every particle of the brick; a kernel block
// stages it in shared memory once, each window cell padded to an even number of slots.
// Each particle keeps its Verlet list as 16-bit window indices of its brick, in blocks
// of 8 entries (16 bytes): block k of particle i at entries [(k * cap + i) * 8, +8),
// padded with the window's sentinel slot wmax - 1 (a particle far away).
constexpr int kBrickMax = 4;  // cells per brick edge
struct BrickView {
  int on;                  // the brick path is in use
  int b[3];                // brick extent in cells
  int nb[3];               // bricks per dimension
  int nbricks;
  int wmax;                // window slots of the shared-memory stage (sentinel included)
  uint16_t* nl;            // Kb * cap entries
  int Kb;                  // entries per particle (multiple of 8)
};

struct DevView {
  ParticleArrays* pa;     // device: pa[0] current arrays, pa[1] target of the re-sort
  int n;                  // particles
  int cap;                // allocated rows
  double L[3], invL[3], halfL[3];
  double cellSize[3], invCellSize[3];
  int nc[3];              // inner cells per dim
  int hci;                // halfCellInt: Verlet candidates from cells within hci cells
  int ncells;
  double fixScale[3];     // 2^32 / L_d   (double -> box-wrapped int32)
  float fixUnit[3];       // L_d / 2^32   (int32 difference -> float length)
  int4* posq;             // box-wrapped int32 coordinates + type
  float4* xrel;           // FP32 position relative to its cell origin at the last re-sort
  int32_t* pcell;         // reference cell of each sorted particle
  int32_t* cellStart;     // ncells + 1
  int32_t* nl;            // K * cap, blocks of 8: entry (k, i) at ((k/8)*cap + i)*8 + k%8
  int32_t* nn;            // neighbour count per particle
  int K;                  // neighbour capacity
  long long* ffix;        // 3*cap pair+bond force, int64 2^-32 fixed point (mixed)
  double* f64;            // 3*cap pair+bond force (FP64 path)
  double* ftot;           // 3*cap total force after the aftCalcF extensions
  int64_t idMin;          // dense id map base
  int idSpan;             // dense id map size
  int32_t* id2idx;        // idSpan: sorted index of id, -1 if absent
  int32_t* bondStart;     // idSpan + 1, CSR of bond partners by id - idMin
  int64_t* bondPartner;   // partner ids
  uint8_t* langExcl;      // idSpan: 1 if the Langevin thermostat skips this id
  uint8_t* halo;          // idSpan: 1 for a copy of another domain's particle (or null)
  int32_t* exclStart;     // idSpan + 1, Verlet-list exclusions by id (or null)
  int64_t* exclIds;
  const LJPair* lj;       // ntypes*ntypes FP64 table (device)
  const LJPairF* ljf;     // float copy for the mixed kernel
  int ntypes;
  int ljSingle;           // only pair (0,0) is set
  int ljCapped;           // some pair uses LennardJonesCapped
  const TabDesc* tabs;    // tabulated potentials (device), coefficients in tabCoef
  const double* tabCoef;
  const int32_t* tabPair; // tabNT*tabNT: table of the type pair on the Verlet list, -1 none
  int tabNT;              // 0: no tabulated pair interaction
  int tabBond;            // table of the fixed pair list, -1 none
  int tabAngle;           // TabulatedAngular table of the fixed triple list, -1 none
  MlpDev mlp;             // learned CG pair potential on the Verlet list (mlp.on)
  const int64_t* triples; // 3 * ntriples ids (p1, p2 centre, p3)
  int ntriples;
  const int32_t* tripStart; // idSpan + 1: CSR of the triples a particle belongs to, by id
  const int32_t* tripEntry; // triple index * 4 + role (0 p1, 1 centre, 2 p3)
  double* tripF;          // 6 * ntriples: force12, force32 of each triple
  CosineParams cosine;
  BrickView brick;        // brick path (brick.on)
  unsigned* err;          // device error word
  DevCounters* ctr;       // step-loop state
};

struct RebuildScratch {
  int32_t* cellOf;    // cap: cell of particle (unsorted order)
  int32_t* slot;      // cap: arrival slot inside its cell
  int32_t* cellCount; // ncells
  int32_t* perm;      // cap: sorted position -> old row
  int32_t* tileSum;   // scan_tiles(ncells): per-tile sums / offsets of the cell scan
};

// launchers (espp_kernels.cu)
void launch_fold_bin(const DevView& d, RebuildScratch& s, bool fold, cudaStream_t st);
void launch_sort_cells(const DevView& d, RebuildScratch& s, cudaStream_t st);
void launch_gather(const DevView& d, const RebuildScratch& s, cudaStream_t st);
void launch_id_map(const DevView& d, cudaStream_t st);
// Verlet list in the global form; fresh: the particles were binned at their current
// positions (the run form may then be used).
void launch_build_nl(const DevView& d, double cutsq, bool fresh, cudaStream_t st);
void launch_posq(const DevView& d, cudaStream_t st);
void launch_xrel(const DevView& d, cudaStream_t st);
void launch_forces(const DevView& d, bool mixed, const FENEParams& fene, int tpp,
                   cudaStream_t st);
struct IntegrateArgs {
  int do_i2, do_i1, langevin, capMode, storeFtot, phase, mixed;
  int fromCounters;  // step from ctr->step; final step (i2 only, store F) when remaining==0
  double dt, pref1, pref2;
  double cap[3];
  uint64_t seed;
  int64_t step;
};
// sustained FP32 FMA throughput of the device (TFLOP/s), scalar or packed, whichever is higher
double measure_fp32_tflops(int nsm, cudaStream_t st);
void launch_wait_selftest(unsigned* err, long long spins, unsigned long long* out,
                          cudaStream_t st);
void launch_integrate(const DevView& d, const IntegrateArgs& a, cudaStream_t st);
// maxDist += sqrt(max |dx|^2); flag = maxDist > skinHalf
void launch_decide(const DevView& d, double skinHalf, cudaStream_t st);
// graph form: also advances ctr->step / ctr->remaining and sets the conditionals
void launch_decide_graph(const DevView& d, double skinHalf, cudaGraphConditionalHandle hIf,
                         cudaGraphConditionalHandle hWhile, cudaStream_t st);
// observables: out[0..6] = (scalar, tensor xx yy zz xy xz yz); deterministic reductions
void launch_lj_observables(const DevView& d, double* partials, int nblocks, double* out,
                           int energy, cudaStream_t st);
void launch_fene_observables(const DevView& d, const FENEParams& fene, double* partials,
                             int nblocks, double* out, int energy, cudaStream_t st);
// pair-distance histogram (integer counts, accumulated into hist) for RadialDistrF
void launch_conf_gather(const DevView& d, const int64_t* ids, int64_t n, int key, double* dst,
                        cudaStream_t st);
int msd_blocks(int64_t n);
void launch_msd(const double* snap, int64_t n, int M, double* partial, cudaStream_t st);
void launch_chain_com(const double* snap, int64_t n, int M, int L, int64_t nch, double* com,
                      cudaStream_t st);
void launch_rdf(const DevView& d, int rdfN, double dr, unsigned long long* hist,
                cudaStream_t st);
// angular forces (per triple, then gathered per particle) added to the force output
void launch_angle_forces(const DevView& d, bool mixed, cudaStream_t st);
// kind 0: interaction::Cosine, 1: TabulatedAngular
void launch_angle_observables(const DevView& d, double* partials, int nblocks, double* out,
                              int energy, int kind, cudaStream_t st);
// tabulated pair and bond forces, added to the main kernel's output
void launch_force_tab(const DevView& d, bool mixed, cudaStream_t st);
void launch_tab_observables(const DevView& d, int bond, double* partials, int nblocks,
                            double* out, int energy, cudaStream_t st);
void launch_kinetic(const DevView& d, double* partials, int nblocks, double* out,
                    cudaStream_t st);
void launch_kinetic_tensor(const DevView& d, double* partials, int nblocks, double* out,
                           cudaStream_t st);
// sum m v^2 (out[0]) and count (out[1]) over the particles of the types in typeMask
void launch_kinetic_types(const DevView& d, unsigned long long typeMask, double* partials,
                          int nblocks, double* out, cudaStream_t st);
// Verlet pair export: counts per particle (pairs with id_j > id_i), then the pairs.
void launch_pair_count(const DevView& d, int32_t* counts, cudaStream_t st);
void launch_pair_write(const DevView& d, const int64_t* offsets, int64_t* out,
                       cudaStream_t st);
// order-independent digest of the Verlet pair set: out[0..4) = count, sum, xor, sum2
void launch_pair_digest(const DevView& d, unsigned long long* partials, int nblocks,
                        unsigned long long* out, cudaStream_t st);
// brick path (espp_brick.cu)
void launch_build_brick(const DevView& d, double cutsq, cudaStream_t st);
void launch_forces_brick(const DevView& d, bool mixed, const FENEParams& fene, cudaStream_t st);
void launch_lj_observables_brick(const DevView& d, double* partials, int nblocks, double* out,
                                 int energy, cudaStream_t st);
void launch_pair_count_brick(const DevView& d, int32_t* counts, cudaStream_t st);
void launch_pair_write_brick(const DevView& d, const int64_t* offsets, int32_t* fill,
                             int64_t* out, cudaStream_t st);
void launch_pair_digest_brick(const DevView& d, unsigned long long* partials,
                              unsigned long long* out, cudaStream_t st);
// shared memory (bytes) a brick window of wmax entries needs: FP32 and FP64 stages
size_t brick_smem_f32(int wmax);
size_t brick_smem_f64(int wmax);
size_t brick_smem_limit();

// float copy of an LJ table for the mixed-precision kernel
void make_float_table(const LJTable& t, LJPairF* out);
int observable_blocks(int n);
int scan_tiles(int ncells);
void launch_set_by_id(const DevView& d, int n, const int64_t* ids, const double* pos,
                      const double* vel, const int32_t* img, cudaStream_t st);
void launch_get_by_id(const DevView& d, int n, const int64_t* ids, double* pos, double* vel,
                      double* force, int32_t* img, cudaStream_t st);

}  // namespace espp
