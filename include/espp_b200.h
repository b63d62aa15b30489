/*
 * espp_b200.h - C ABI of the B200 short-range MD step (cell binning, Verlet list,
 * Lennard-Jones / FENE forces, velocity Verlet with Langevin thermostat).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an
 * int status: 0 on success, a negative ESPP_E* code on failure.  The text of the last
 * failure on the calling thread is available through espp_last_error().
 *
 * One espp_system is one simulation box with all of its particles resident on one
 * GPU (the CUDA library, libespp_b200.so).  The same ABI is implemented on the host in
 * FP64 by the test oracle; the two are compared call for call by the parity tests.
 *
 * Each entry point names the ESPResSo++ interface it replaces (paths inside the
 * espressopp/espressopp source tree).  Arrays of 3-vectors are interleaved
 * (x0,y0,z0,x1,...).  Particle identity is the 64-bit particle id of the reference.
 * A handle is not thread safe; calls on one handle must be serialised by the caller.
 */
#ifndef ESPP_B200_H
#define ESPP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ESPP_API __attribute__((visibility("default")))
#else
#define ESPP_API
#endif

typedef struct espp_system espp_system;

/* status codes */
#define ESPP_OK 0
#define ESPP_EINVAL (-1)    /* bad argument (message says which) */
#define ESPP_ESTATE (-2)    /* call not valid in the current state */
#define ESPP_ECUDA (-3)     /* CUDA runtime error */
#define ESPP_ERANGE (-4)    /* value outside the supported range */
#define ESPP_ENOMEM (-5)    /* allocation failed */
#define ESPP_EOVERFLOW (-6) /* a fixed-capacity structure overflowed */
#define ESPP_ETIMEOUT (-7)  /* a bounded device wait gave up */
#define ESPP_ENAN (-8)      /* non-finite particle coordinate */

/* precision modes */
#define ESPP_PREC_FP64 0  /* all-FP64 pair forces (plain form) */
#define ESPP_PREC_MIXED 1 /* FP32 pair forces, int64 2^-32 fixed-point sums, FP64 integrator */

/* interaction kinds for the observable calls */
#define ESPP_IA_LJ 0   /* VerletListLennardJones */
#define ESPP_IA_FENE 1 /* FixedPairListFENE */
#define ESPP_IA_TAB_PAIR 2 /* VerletListTabulated */
#define ESPP_IA_TAB_BOND 3 /* FixedPairListTabulated */
#define ESPP_IA_MLP 4      /* learned coarse-grained pair potential (espp_mlp_*) */
#define ESPP_IA_COSINE 5   /* FixedTripleListCosine */
#define ESPP_IA_TAB_ANGLE 6 /* FixedTripleListTabulatedAngular */

/* interpolation types of interaction::Tabulated (src/interaction/Tabulated.cpp:49-67) */
#define ESPP_TAB_LINEAR 1
#define ESPP_TAB_AKIMA 2
#define ESPP_TAB_CUBIC 3

/* force-capping modes (integrator::CapForce) */
#define ESPP_CAP_OFF 0
#define ESPP_CAP_ABS 1       /* |F| <= cap[0] */
#define ESPP_CAP_COMPONENT 2 /* |F_d| <= cap[d] */

ESPP_API int espp_abi_version(void);

/* Copies the last error message of this thread (NUL terminated, truncated to cap) and
 * returns its full length. */
ESPP_API size_t espp_last_error(char* buf, size_t cap);

/* ---- System + bc::OrthorhombicBC + storage::DomainDecomposition -------------------
 * Replaces System (src/System.cpp:40-105), OrthorhombicBC::setBoxL
 * (src/bc/OrthorhombicBC.cpp:40-50) and the DomainDecomposition constructor
 * (src/storage/DomainDecomposition.cpp:70-85) on one node: nodeGrid = (1,1,1), cell
 * grid as given (tools/decomp.py:322-342 computes it), at least 3 cells a dimension;
 * halfCellInt 1 (espp_set_half_cell_int sets another). */
ESPP_API int espp_system_create(const double box[3], double skin, const int32_t cell_grid[3],
                       int32_t precision, uint64_t seed, espp_system** out);
ESPP_API int espp_system_destroy(espp_system* s);
/* System::setSkin (src/System.cpp:75-93). */
ESPP_API int espp_set_skin(espp_system* s, double skin);

/* Storage::addParticle + property setters (src/storage/Storage.cpp:285-313,
 * src/storage/Storage.py:233-330).  type/mass/vel may be NULL (defaults 0, 1.0, 0). */
ESPP_API int espp_add_particles(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                       const double* mass, const double* pos, const double* vel);
/* Storage::decompose (src/storage/Storage.cpp:598-604): fold, re-bin, rebuild lists. */
ESPP_API int espp_decompose(espp_system* s);
ESPP_API int espp_num_particles(espp_system* s, int64_t* n);
/* Storage::lookupRealParticle + Particle accessors (src/Particle.hpp:44-410) for n ids.
 * Any of pos/vel/force/image may be NULL. */
ESPP_API int espp_get_particles(espp_system* s, int64_t n, const int64_t* ids, double* pos,
                       double* vel, double* force, int32_t* image);
/* Particle setters for existing ids (pos/vel may be NULL). */
ESPP_API int espp_set_particles(espp_system* s, int64_t n, const int64_t* ids, const double* pos,
                       const double* vel);
/* Image counts (3 n int32) of existing ids: Storage.modifyParticle(pid, 'img', value)
 * (src/storage/Storage.py:385).  Positions are left as they are. */
ESPP_API int espp_set_images(espp_system* s, int64_t n, const int64_t* ids, const int32_t* img);

/* ---- VerletList (src/VerletList.cpp:196-270, :274-450) ----------------------------
 * cutoff is the interaction cutoff; the list holds pairs with |d| <= cutoff + skin.
 * excl_pairs: nexcl id pairs never listed (VerletList::exclude, :480-485). */
ESPP_API int espp_vl_create(espp_system* s, double cutoff, int64_t nexcl, const int64_t* excl_pairs);
ESPP_API int espp_vl_rebuild(espp_system* s);
/* VerletList::totalSize (:454-462). */
ESPP_API int espp_vl_size(espp_system* s, int64_t* npairs);
/* getAllPairs as unordered id pairs, each written (min id, max id), sorted
 * lexicographically (testsuite/verlet_list_buffer/verlet_list_buffer.py sort_pairs).
 * Writes at most cap pairs (2*cap int64); *npairs receives the total. */
ESPP_API int espp_vl_pairs(espp_system* s, int64_t cap, int64_t* pairs, int64_t* npairs);
ESPP_API int espp_vl_builds(espp_system* s, int64_t* builds);
/* Order-independent digest of the Verlet pair set, each unordered pair once by id:
 * out[0] the number of pairs, out[1] the wrapping sum and out[2] the xor of the 64-bit
 * hash h = mix(mix(smaller id) ^ larger id) (mix: the splitmix64 finaliser), out[3] the
 * wrapping sum of mix(h).  Equal pair sets give equal digests whatever the list order;
 * it compares lists of millions of pairs without exporting them (the reference's
 * VerletList::getAllPairs, VerletList.cpp:515-536, exports the pairs themselves). */
ESPP_API int espp_vl_digest(espp_system* s, uint64_t out[4]);

/* ---- interaction::LennardJones / LennardJonesCapped on the Verlet list -------------
 * VerletListInteractionTemplate::setPotential (src/interaction/
 * VerletListInteractionTemplate.hpp:65-78) with LennardJones(eps, sig, rc, shift)
 * (src/interaction/LennardJones.hpp:56-87).  caprad > 0 selects LennardJonesCapped
 * (src/interaction/LennardJonesCapped.hpp:80-160).  shift is the final energy shift. */
ESPP_API int espp_lj_set(espp_system* s, int32_t type1, int32_t type2, double epsilon, double sigma,
                double cutoff, double shift, double caprad);

/* ---- FixedPairList + interaction::FENE --------------------------------------------
 * FixedPairList::add (src/FixedPairList.cpp:88-141): pairs are id pairs. */
ESPP_API int espp_bonds_add(espp_system* s, int64_t n, const int64_t* pairs);
ESPP_API int espp_bonds_size(espp_system* s, int64_t* n);
/* FixedPairList::remove (src/FixedPairList.cpp:317-324): empties the bond list. */
ESPP_API int espp_bonds_clear(espp_system* s);
/* FixedPairListFENE(system, fpl, FENE(K, r0, rMax, cutoff, shift))
 * (src/interaction/FENE.hpp:35-115, src/interaction/FENE.cpp:45-53). */
ESPP_API int espp_fene_set(espp_system* s, double K, double r0, double rmax, double cutoff,
                  double shift);
/* FixedPairList::getLongtimeMaxBondSqr (src/FixedPairList.cpp:82): the longest bond^2
 * seen by any force pass since the system was made or the maximum was last reset
 * (every force pass raises it, FixedPairListInteractionTemplate.hpp:145-150); 0 before
 * the first force pass. */
ESPP_API int espp_bonds_max_sqr(espp_system* s, double* maxsq);
/* FixedPairList::resetLongtimeMaxBondSqr (src/FixedPairList.cpp:86): sets it to 0. */
ESPP_API int espp_bonds_reset_max(espp_system* s);

/* ---- FixedTripleList + interaction::Cosine ---------------------------------------------
 * FixedTripleList::add (src/FixedTripleList.cpp): triples of ids (p1, p2, p3), p2 the
 * centre.  FixedTripleListCosine(system, ftl, Cosine(K, theta0))
 * (src/interaction/Cosine.hpp:38-125, FixedTripleListInteractionTemplate.hpp:121-333):
 * E = K (1 + cos(theta - theta0)). */
ESPP_API int espp_triples_add(espp_system* s, int64_t n, const int64_t* triples);
ESPP_API int espp_triples_size(espp_system* s, int64_t* n);
/* FixedTripleList::remove (src/FixedTripleList.py:97-100): empties the triple list. */
ESPP_API int espp_triples_clear(espp_system* s);
ESPP_API int espp_cosine_set(espp_system* s, double K, double theta0);

/* ---- interaction::Tabulated -----------------------------------------------------------
 * Table files as InterpolationLinear/Akima/Cubic::readFile read them
 * (src/interaction/InterpolationLinear.cpp readFile; same in the Akima and Cubic
 * variants): every line whose first three fields parse as numbers (sscanf "%lg %lg %lg")
 * is one entry (r, energy, force); other lines are skipped.  Writes at most cap
 * entries, *n receives the count.  Fewer than 2 entries is ESPP_EINVAL ("illegal file
 * for tabulated potential"), an unreadable file ESPP_EINVAL. */
ESPP_API int espp_tab_read(const char* path, int64_t cap, double* r, double* energy,
                           double* force, int64_t* n);
/* Interpolation::getEnergy / getForce (src/interaction/InterpolationLinear.hpp,
 * InterpolationAkima.hpp, InterpolationCubic.hpp) of the table (r, e, f) of n entries at
 * m distances x, on the host: the scalar evaluation behind Tabulated's computeEnergy /
 * computeForce.  Either output may be NULL. */
ESPP_API int espp_tab_eval(int32_t itype, int64_t n, const double* r, const double* e,
                           const double* f, int64_t m, const double* x, double* energy,
                           double* force);
/* VerletListTabulated::setPotential(type1, type2, Tabulated(itype, table, cutoff))
 * (src/interaction/Tabulated.cpp:85-95, Tabulated.hpp:43-115): the pair interacts through
 * the table on the system's Verlet list.  shift is the final energy shift (0 unless the
 * caller sets one).  Replaces an earlier table of the same type pair. */
ESPP_API int espp_tab_pair_set(espp_system* s, int32_t type1, int32_t type2, int32_t itype,
                               int64_t n, const double* r, const double* e, const double* f,
                               double cutoff, double shift);
/* FixedPairListTabulated(system, fpl, Tabulated(itype, table, cutoff))
 * (src/interaction/Tabulated.cpp:147-158): the bonds of the system's fixed pair list
 * interact through the table (in addition to FENE when that is set too). */
ESPP_API int espp_tab_bond_set(espp_system* s, int32_t itype, int64_t n, const double* r,
                               const double* e, const double* f, double cutoff, double shift);
/* FixedTripleListTabulatedAngular(system, ftl, TabulatedAngular(itype, table))
 * (src/interaction/TabulatedAngular.hpp:75-113): the triples of the system's fixed triple
 * list interact through E(theta) of the table (theta in radians, f = -dE/dtheta), with
 * force12 = a11 d12 + a12 d32, force32 = a22 d32 + a12 d12, a = f(acos c) / sqrt(1 - c^2),
 * a11 = a c / |d12|^2, a12 = -a / (|d12| |d32|), a22 = a c / |d32|^2.  Replaces an
 * earlier angle table; acts in addition to interaction::Cosine when that is set too. */
ESPP_API int espp_tab_angle_set(espp_system* s, int32_t itype, int64_t n, const double* theta,
                                const double* e, const double* f);

/* ---- integrator::VelocityVerlet + extensions ---------------------------------------
 * MDIntegrator::setTimeStep (src/integrator/MDIntegrator.cpp:53-60). */
ESPP_API int espp_integrator_set(espp_system* s, double dt);
/* MDIntegrator step counter (read / write). */
ESPP_API int espp_step_get(espp_system* s, int64_t* step);
ESPP_API int espp_step_set(espp_system* s, int64_t step);
/* LangevinThermostat gamma/temperature/exclusions (src/integrator/
 * LangevinThermostat.cpp:41-214).  gamma == 0 and temperature == 0 disables it.  The
 * noise is Philox4x32-10 keyed on (seed, particle id) with counter (step, phase). */
ESPP_API int espp_langevin_set(espp_system* s, int32_t enabled, double gamma, double temperature,
                      int64_t nexcl, const int64_t* excl_ids);
/* CapForce (src/integrator/CapForce.cpp:34-200). */
ESPP_API int espp_capforce_set(espp_system* s, int32_t mode, const double cap[3]);
/* VelocityVerlet::run (src/integrator/VelocityVerlet.cpp:63-169). */
ESPP_API int espp_run(espp_system* s, int64_t nsteps);
/* VelocityVerlet::getNumResorts (:246). */
/* ---- spatial decomposition: one system per domain -------------------------------------
 * DomainDecomposition over several domains (src/storage/DomainDecomposition.cpp:1031-1158
 * migration, :1243-1391 ghost frames; one domain per GPU).  Each domain's system holds the
 * particles it owns and halo copies of the particles of the neighbouring domains' boundary
 * cells; halo particles are partners only: not integrated, not thermostatted, and skipped
 * as the first particle of every observable, so that energies, virials, kinetic sums and
 * pair sets of all domains add up to the undecomposed system's (a pair with a halo partner
 * is counted by the domain owning the smaller id).  Angles, the learned potential and the
 * RDF are refused while halo particles are present.
 * espp_dd_load replaces every particle of the system (positions as integrated, not
 * folded: the next step re-sorts them; halo[i] != 0 marks halo copies).
 * espp_dd_set_halo_positions moves halo copies to their owners' positions (no re-sort).
 * A run of nsteps is espp_dd_run_begin (re-sort if loaded, start-of-run force with the
 * Langevin heat-up, integrate1 of step 0), nsteps x espp_dd_step (re-sort when resort or
 * after a load, force, aftCalcF + integrate2, integrate1 of the next step), then
 * espp_dd_run_end; begin and step return the step's largest displacement sqrt(max |dx|^2)
 * over the owned particles (0 after the last step), from which the host decides the next
 * re-sort (VelocityVerlet.cpp:63-169). */
ESPP_API int espp_dd_load(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                          const double* mass, const double* pos, const double* vel,
                          const int32_t* img, const uint8_t* halo);
ESPP_API int espp_dd_set_halo_positions(espp_system* s, int64_t n, const int64_t* ids,
                                        const double* pos);
/* The memory space of the library's particle arrays: 0 host memory (the CPU oracle),
 * 1 device memory of the system's GPU (the CUDA library). */
ESPP_API int espp_memory_space(int32_t* kind);
/* Halo refresh without host round trips: ids (n) and pos (3n doubles) lie in the
 * library's memory space (device arrays for the CUDA library), so the positions can move
 * between domains by NCCL or a device copy.  espp_dd_read_positions copies the positions
 * of the listed particles out, espp_dd_write_halo moves halo copies to the given
 * positions; both return when the copy is complete. */
ESPP_API int espp_dd_read_positions(espp_system* s, int64_t n, const int64_t* ids,
                                    double* pos);
ESPP_API int espp_dd_write_halo(espp_system* s, int64_t n, const int64_t* ids,
                                const double* pos);
ESPP_API int espp_dd_run_begin(espp_system* s, int64_t nsteps, double* maxd);
ESPP_API int espp_dd_step(espp_system* s, int32_t resort, double* maxd);
ESPP_API int espp_dd_run_end(espp_system* s);

ESPP_API int espp_num_resorts(espp_system* s, int64_t* n);
/* VelocityVerlet::loadTimers (:206-218): run, pair, FENE, angle, comm1, comm2, int1,
 * int2, resort, other (seconds). */
ESPP_API int espp_timers(espp_system* s, double t[10]);

/* ---- batched replicas -------------------------------------------------------------
 * MultiSystem / ParallelTempering on one GPU (src/MultiSystem.py:105-125,
 * src/ParallelTempering.py:78-203): n independent systems on the same device stepped by
 * one graph launch that holds one step loop per system, with no dependencies between
 * them, so the replicas run concurrently and each keeps its own re-sort schedule.  The
 * systems stay owned by the caller and must outlive the batch; results per system are
 * identical to espp_run on that system alone. */
typedef struct espp_batch espp_batch;
ESPP_API int espp_batch_create(espp_system* const* systems, int32_t n, espp_batch** out);
ESPP_API int espp_batch_destroy(espp_batch* b);
ESPP_API int espp_batch_run(espp_batch* b, int64_t nsteps);
/* Device time of the last espp_batch_run's graph launch (ms). */
ESPP_API int espp_batch_last_run_ms(espp_batch* b, double* ms);

/* ---- observables (FP64) --------------------------------------------------------
 * Interaction::computeEnergy / computeVirial / computeVirialTensor
 * (VerletListInteractionTemplate.hpp:201-331, FixedPairListInteractionTemplate.hpp:
 * 207+, 400-440).  Tensor order xx, yy, zz, xy, xz, yz (src/Tensor.hpp:125-133). */
ESPP_API int espp_energy(espp_system* s, int32_t which, double* e);
ESPP_API int espp_virial(espp_system* s, int32_t which, double* w);
ESPP_API int espp_virial_tensor(espp_system* s, int32_t which, double w[6]);
/* sum m v^2 over real particles and their count (analysis/Temperature.hpp:57-125). */
ESPP_API int espp_kinetic(espp_system* s, double* sum_mv2, int64_t* n);
/* sum over real particles of mass * Tensor(v, v) (analysis/PressureTensor.hpp:60-70):
 * out = (xx, yy, zz, xy, xz, yz), each m (v_a v_b). */
ESPP_API int espp_kinetic_tensor(espp_system* s, double out[6]);
/* Sum of m v^2 and count over the particles whose type t (0 <= t < 64) has bit t set in
 * type_mask: Temperature::compute_real with add_type (src/analysis/Temperature.hpp:57-125,
 * valid_type_ids). */
ESPP_API int espp_kinetic_types(espp_system* s, uint64_t type_mask, double* sum_mv2, int64_t* n);

/* analysis::RadialDistrF::computeArray(rdfN) (src/analysis/RadialDistrF.cpp:47-150): histogram
 * of all pair distances (minimum image) in rdfN bins of width dr = L_y / (2 rdfN), each
 * bin divided by 2 pi dr rho N ((i + 1/2)^2 dr^2 + dr^2 / 12).  out receives rdfN values. */
ESPP_API int espp_rdf(espp_system* s, int32_t rdfN, double* out);

/* Snapshots of tracked particles kept on the device: analysis::ConfigsParticleDecomp
 * (src/analysis/ConfigsParticleDecomp.hpp:61-230, ConfigsParticleDecomp.cpp:43-206) and its
 * MeanSquareDispl (src/analysis/MeanSquareDispl.cpp).  A snapshot holds, for each tracked id
 * in the order given at creation (ascending, as the reference's id map iterates), the
 * position, the velocity or the unfolded position x + image * L (ESPP_CONF_*).  The handle
 * refers to its system and must be destroyed before it. */
typedef struct espp_confs espp_confs;
#define ESPP_CONF_POSITION 0
#define ESPP_CONF_VELOCITY 1
#define ESPP_CONF_UNFOLDED 2
ESPP_API int espp_confs_create(espp_system* s, int32_t key, int64_t n, const int64_t* ids,
                               espp_confs** out);
ESPP_API int espp_confs_destroy(espp_confs* c);
/* ConfigsParticleDecomp::gather (ConfigsParticleDecomp.cpp:70-142): appends the current
 * state.  ESPP_ESTATE if a tracked id is not in the system. */
ESPP_API int espp_confs_gather(espp_confs* c);
/* Appends a snapshot given by the caller (gatherFromFile, :144-206): 3 n values x y z per
 * tracked id, in the tracked order. */
ESPP_API int espp_confs_push(espp_confs* c, const double* xyz);
ESPP_API int espp_confs_size(espp_confs* c, int32_t* m);
ESPP_API int espp_confs_clear(espp_confs* c);
/* Snapshot m as 3 n values (ConfigsParticleDecomp::getConf); ESPP_ERANGE if m is outside. */
ESPP_API int espp_confs_get(espp_confs* c, int32_t m, double* xyz);
/* MeanSquareDispl::compute (MeanSquareDispl.cpp:42-141) over the M snapshots:
 * out[m] = (sum_{t < M-m} sum_i |r_i(t) - r_i(t+m)|^2 / (M - m)) / (6 N), m = 0 .. M-1. */
ESPP_API int espp_msd(espp_confs* c, double* out);
/* MeanSquareDispl::computeG3 (MeanSquareDispl.cpp:248-430): the same over the centres of
 * mass of chains of chainlength consecutive tracked particles, each taken relative to the
 * mean of that snapshot's chain centres; out[m] = (sum / (6 C)) / (M - m) for C chains. */
ESPP_API int espp_msd_chain_com(espp_confs* c, int32_t chainlength, double* out);

/* Sums of the total force (the force espp_get_particles reports) by particle id, kept on
 * the device across runs and re-sorts: op 0 clears the sums, op 1 adds the current total
 * forces, op 2 copies the sums of the particles ids (3 per particle) to out.  Serves
 * time averages of forces, e.g. mapped forces over a window of steps.  No counterpart in
 * the reference. */
ESPP_API int espp_force_acc(espp_system* s, int32_t op, int64_t n, const int64_t* ids,
                            double* out);

/* ---- learned coarse-grained potential -------------------------------------------------
 * No counterpart in the reference: a many-body pair potential for coarse-grained sites,
 * with interaction::Tabulated as its fallback.  Per particle i a descriptor of 16
 * Gaussian radial basis functions over the Verlet-list partners within rc,
 *   G_i[k] = sum_j exp(-(r_ij - mu_k)^2 / (2 w^2)) (cos(pi r_ij / rc) + 1) / 2,
 *   mu_k = r0 + k w, w = (rc - r0) / 15,
 * normalised as x_i = (G_i - shift) * scale, feeds an MLP 16-64-64-1 with SiLU
 * activations giving the site energy E_i; E = sum_i E_i and F = -grad E.  Parameters
 * (espp_mlp_num_params of them, in the order W1[64][16], b1[64], W2[64][64], b2[64],
 * w3[64], b3) live on the device.  Training is by force matching: espp_mlp_fm_grad
 * evaluates the mean squared force-component error of one configuration against
 * reference forces and adds its gradient to the model's accumulator;
 * espp_mlp_adam_step applies Adam (gradient times gscale) and clears the accumulator. */
typedef struct espp_mlp espp_mlp;
ESPP_API int espp_mlp_create(double rc, double r0, espp_mlp** out);
ESPP_API int espp_mlp_destroy(espp_mlp* m);
/* Site network arithmetic: 1 (default) BF16 operands on the tensor cores (tcgen05) with
 * FP32 accumulation, 0 FP32 on the CUDA cores.  The mode applies to the force pass and to
 * the weight-gradient products of espp_mlp_fm_grad (the descriptor, the tangent and the
 * bias sums stay FP32). */
ESPP_API int espp_mlp_set_mode(espp_mlp* m, int32_t tensor_cores);
ESPP_API int espp_mlp_num_params(int64_t* n);
ESPP_API int espp_mlp_set_params(espp_mlp* m, int64_t n, const double* theta);
ESPP_API int espp_mlp_get_params(espp_mlp* m, int64_t n, double* theta);
ESPP_API int espp_mlp_set_norm(espp_mlp* m, const double shift[16], const double scale[16]);
/* Adds the model as an interaction of s on its Verlet list (cutoff >= rc); NULL removes
 * it.  The model is not owned by the system and must outlive the attachment. */
ESPP_API int espp_mlp_attach(espp_system* s, espp_mlp* m);
/* Descriptors G (16 per particle) of the particles ids, in that order. */
ESPP_API int espp_mlp_descriptors(espp_system* s, int64_t n, const int64_t* ids, double* G);
/* Loss and gradient on the current configuration against reference forces fref (3 per
 * particle, given in the order of ids, every particle once).  grad (optional) receives
 * this configuration's gradient; the model accumulator receives it too. */
ESPP_API int espp_mlp_fm_grad(espp_system* s, int64_t n, const int64_t* ids,
                              const double* fref, double* loss, double* grad);
ESPP_API int espp_mlp_adam_step(espp_mlp* m, double lr, double beta1, double beta2, double eps,
                                double gscale);

/* Same result as espp_energy (identical kernels and reduction order), but the call
 * allocates no device memory: the per-block partial sums live in a statically sized
 * array inside the library instead of a buffer obtained with cudaMalloc.  No
 * counterpart exists in the reference.  It is meant for callers that may not allocate
 * GPU memory themselves or have a library do it for them: hosts whose device memory
 * is owned by another allocator (a framework's pool or caching allocator, or a fixed
 * memory budget), and time-critical loops where a first-use cudaMalloc or cudaFree
 * would synchronise the device.
 *   - Limit: at most 8,388,608 particles (32768 reduction blocks of 256); more gives
 *     ESPP_ERANGE.  The static array (1.8 MB) is held on every GPU that loads the
 *     library until the process exits.
 *   - The system must be ready: particles sorted and, for ESPP_IA_LJ, the Verlet list
 *     built (after espp_decompose, espp_run or espp_energy); otherwise ESPP_ESTATE.
 *   - The first call on a device looks up the array's device address with that device
 *     current; make that first call before any stream capture on that device.  The
 *     address is kept per device together with the id of the CUDA context it belongs
 *     to; after a device reset (or a released and re-retained primary context) the next
 *     call looks it up again, so that call too should come before any stream capture.
 *   - All calls share the one array, which keeps the last call's contents; calls that
 *     overlap on the GPU (two systems on different streams or threads) race. */
ESPP_API int espp_energy_noalloc(espp_system* s, int32_t which, double* e);

/* ---- measurement ---------------------------------------------------------------
 * No reference counterpart (the reference times phases with esutil::WallTimer,
 * VelocityVerlet.cpp:171-232).  With profiling on, run() steps on the host-driven loop
 * and brackets each phase with CUDA events on the system's stream: ms[0] pair/bond
 * force kernel, ms[1] integrator kernel, ms[2] re-sort (fold, bin, sort, gather),
 * ms[3] rebuild decision, ms[4] Verlet build, ms[5..7] unused; launches[] counts the
 * kernels of each phase (also without profiling).  espp_set_profiling resets both. */
ESPP_API int espp_set_profiling(espp_system* s, int32_t on);
ESPP_API int espp_profile(espp_system* s, double ms[8], int64_t launches[8]);
/* Threads per particle of the force kernel (1, 2, 4 or 8; default 4, or the
 * environment variable ESPP_B200_TPP).  The FP32 partial sums of the threads are combined
 * in int64 fixed point, so the value changes the rounding of the mixed-precision forces
 * (within the 1e-5 error budget) but not their determinism for a fixed setting.
 * No reference counterpart (tuning of the GPU kernel). */
ESPP_API int espp_set_tpp(espp_system* s, int32_t tpp);

/* Sustained FP32 FMA throughput of the current device in TFLOP/s (a probe kernel of
 * independent scalar and packed f32x2 FMA chains, the higher of the two), for the FLOP
 * side of the step's roofline.  No reference counterpart. */
ESPP_API int espp_fp32_peak(double* tflops);
/* Runs the tensor-core kernels' failure path on purpose: one CTA holds TMEM and waits,
 * for at most `spins` tries (1 to 2^20), on an mbarrier that nothing arrives on, then
 * releases the TMEM and returns; *ns (may be NULL) receives the nanoseconds the wait took.
 * Returns ESPP_ETIMEOUT ("a bounded wait inside a kernel ran out") when the wait gave up,
 * as it must, and leaves the system usable.  No reference counterpart. */
ESPP_API int espp_selftest_bounded_wait(espp_system* s, int64_t spins, double* ns);
/* Times the force kernel on the current particle state for 1, 2, 4 and 8 threads per
 * particle (3 launches each, CUDA events), keeps the fastest and returns it; ms[c] (may
 * be NULL) receives the mean launch time of candidate c. */
ESPP_API int espp_autotune(espp_system* s, int32_t* best_tpp, double ms[4]);
/* DomainDecomposition's halfCellInt (src/storage/DomainDecomposition.cpp:325-357,
 * tools/decomp.py:322): the cell grid given to espp_system_create is the fine grid, and a
 * particle's Verlet candidates come from the cells within h cells in each direction (a
 * (2h + 1)^3 stencil).  1 .. 4, the grid at least 2h + 1 cells a dimension; set before
 * any particle is added (ESPP_ESTATE otherwise).  h > 1 takes the global list form. */
ESPP_API int espp_set_half_cell_int(espp_system* s, int32_t h);
/* List layout of the Verlet list and pair kernels (tuning of the GPU kernels; no
 * reference counterpart).  form 0: one global list per particle (sorted indices) built
 * by runs of 32 particles of a row of cells (one warp per cell where cells were binned
 * at other positions), tpp (1, 2, 4, 8) threads per particle in the force kernel;
 * form 2: the same global list built by brick windows (brick[3] cells per brick edge,
 * 1..4, or all 0 to choose from the density); form 1: brick windows for the build and
 * the force kernels, one thread per particle with its list as 16-bit window indices.
 * Forms 1 and 2 need grids of at least 2 cells per dimension; form 1 serves
 * Lennard-Jones (plain or capped), FENE bonds and exclusions, tabulated and learned pair
 * potentials use the global list.  All forms give the reference's pair set; the
 * mixed-precision forces differ in rounding (within the 1e-5 budget).  The list is
 * rebuilt at the current positions (not counted as a build). */
ESPP_API int espp_set_layout(espp_system* s, int32_t form, int32_t tpp, const int32_t brick[3]);
/* out = (form, tpp, brick extent x, y, z) of the list in use. */
ESPP_API int espp_get_layout(espp_system* s, int32_t out[5]);
/* Times each candidate layout on the current particle state (one list build and 3
 * force launches each, CUDA events), keeps the one with the smallest force time plus
 * build time / steps_per_build (<= 0: 10), and returns it in best (as espp_get_layout).
 * table (may be NULL) receives up to cap rows (form, tpp, bx, by, bz, force ms, build ms,
 * score); ncand the number of candidates timed. */
ESPP_API int espp_autotune_layout(espp_system* s, double steps_per_build, int32_t best[5],
                                  double* table, int32_t cap, int32_t* ncand);
/* Device time of the last espp_run on the system's stream (ms): ms[0] whole call,
 * ms[1] the step loop after the start-of-run force evaluation. */
ESPP_API int espp_last_run_ms(espp_system* s, double ms[2]);
/* Selects the CUDA device for systems created afterwards on the calling thread. */
ESPP_API int espp_select_device(int32_t device);

#ifdef __cplusplus
}
#endif

#endif /* ESPP_B200_H */
