/*
 * lima_abi.h — C-ABI of the B200-native LIMA_MD step engine (quantom_b200).
 *
 * The reference (DanielRJohansen/Quantom, "LIMA_MD") has no plugin or FFI
 * interface: its per-step path sits behind the C++ class Engine
 * (Quantom/Quantom/Engine.cuh:109-208) operating on a Box in CUDA managed
 * memory (Quantom/Quantom/Simulation.cuh:35-92), driven by
 * Environment::run (Quantom/Quantom/Environment.cpp:100-122).  This header is
 * the boundary that replaces it: plain C, plain pointers and sizes, status
 * codes instead of exit(), caller-owned host buffers, library-owned device
 * memory.  The structs below are byte-compatible with the reference's own
 * (sizes in comments; tests/test_layout_and_abi.py checks them against a build of
 * the reference), so the reference's Box arrays can be passed unchanged.
 *
 * Units are the reference's: positions nm, time ns, mass kg/mol, energy J/mol,
 * force J/(mol nm).
 */
#ifndef LIMA_ABI_H
#define LIMA_ABI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Reference layout (Quantom/Quantom/Bodies.cuh, QuantomTypes.cuh,      */
/* Forcefield.cuh).  Capacities are the reference's constants.          */
/* ------------------------------------------------------------------ */
#define LIMA_MAX_COMPOUND_PARTICLES 64        /* Constants.cuh:58 */
#define LIMA_MAX_PAIRBONDS 128                /* Bodies.cuh:300 */
#define LIMA_MAX_ANGLEBONDS 256               /* Bodies.cuh:301 */
#define LIMA_MAX_DIHEDRALS 384                /* Bodies.cuh:302 */
#define LIMA_LJ_IGNORES_MAX 32                /* Bodies.cuh:170 */
#define LIMA_MAX_PARTICLES_IN_BRIDGE 32       /* Constants.cuh:110 */
#define LIMA_MAX_SINGLEBONDS_IN_BRIDGE 32     /* Constants.cuh:111 */
#define LIMA_MAX_ANGLEBONDS_IN_BRIDGE 32      /* Constants.cuh:112 */
#define LIMA_MAX_DIHEDRALBONDS_IN_BRIDGE 32   /* Constants.cuh:113 */
#define LIMA_MAX_ATOM_TYPES 32                /* Forcefield.cuh:12 */
#define LIMA_MAX_COMPOUNDS 255                /* Constants.cuh:88: LJ_Ignores holds uint8 compound ids */
#define LIMA_ATOMTYPE_SOL 0                   /* Forcefield.cuh:15 */

typedef struct { float x, y, z; } lima_float3;                       /* Float3, 12 B */

typedef struct { lima_float3 pos, pos_tsub1; } lima_solvent;          /* Solvent, 24 B */

typedef struct { float b0, kb; uint32_t atom_indexes[2]; } lima_pair_bond;            /* PairBond, 16 B */
typedef struct { float theta_0, k_theta; uint32_t atom_indexes[3]; } lima_angle_bond; /* AngleBond, 20 B */
typedef struct { float phi_0, k_phi; uint8_t n; uint32_t atom_indexes[4]; } lima_dihedral_bond; /* DihedralBond, 28 B */

typedef struct {                                                      /* LJ_Ignores, 65 B */
    uint8_t local_ids[LIMA_LJ_IGNORES_MAX];
    uint8_t compound_ids[LIMA_LJ_IGNORES_MAX];
    uint8_t n_ignores;
} lima_lj_ignores;

typedef struct {                                                      /* CompoundState, 772 B */
    lima_float3 positions[LIMA_MAX_COMPOUND_PARTICLES];
    uint8_t n_particles;
} lima_compound_state;

typedef struct {                                                      /* Compound (LIMA_DEBUGMODE), 24,036 B */
    uint8_t n_particles;
    lima_float3 prev_positions[LIMA_MAX_COMPOUND_PARTICLES];
    lima_float3 forces[LIMA_MAX_COMPOUND_PARTICLES];
    uint8_t atom_types[LIMA_MAX_COMPOUND_PARTICLES];
    uint8_t atom_color_types[LIMA_MAX_COMPOUND_PARTICLES];
    lima_lj_ignores lj_ignore_list[LIMA_MAX_COMPOUND_PARTICLES];
    uint32_t particle_global_ids[LIMA_MAX_COMPOUND_PARTICLES];
    lima_float3 center_of_mass;
    uint16_t n_singlebonds;
    lima_pair_bond singlebonds[LIMA_MAX_PAIRBONDS];
    uint16_t n_anglebonds;
    lima_angle_bond anglebonds[LIMA_MAX_ANGLEBONDS];
    uint16_t n_dihedrals;
    lima_dihedral_bond dihedrals[LIMA_MAX_DIHEDRALS];
    int32_t key_particle_index;
    float confining_particle_sphere;
} lima_compound;

typedef struct { int32_t compound_id, local_id_compound; } lima_particle_ref_compact; /* 8 B */

typedef struct {                                                      /* CompoundBridgeCompact, 2,352 B */
    lima_particle_ref_compact particle_refs[LIMA_MAX_PARTICLES_IN_BRIDGE];
    uint8_t atom_types[LIMA_MAX_PARTICLES_IN_BRIDGE];
    int32_t n_particles;
    uint16_t n_singlebonds;
    lima_pair_bond singlebonds[LIMA_MAX_SINGLEBONDS_IN_BRIDGE];
    uint16_t n_anglebonds;
    lima_angle_bond anglebonds[LIMA_MAX_ANGLEBONDS_IN_BRIDGE];
    uint16_t n_dihedrals;
    lima_dihedral_bond dihedrals[LIMA_MAX_DIHEDRALBONDS_IN_BRIDGE];
} lima_compound_bridge_compact;

typedef struct { float mass, sigma, epsilon; } lima_particle_parameters;                  /* 12 B */
typedef struct { lima_particle_parameters particle_parameters[LIMA_MAX_ATOM_TYPES]; } lima_forcefield; /* 384 B */

/* ------------------------------------------------------------------ */
/* Engine parameters (the reference's compile-time Constants.cuh:6-113  */
/* and Simulation.cuh:152 become runtime values).                       */
/* ------------------------------------------------------------------ */
typedef enum {
    LIMA_OK = 0,
    LIMA_ERR_ARGUMENT = 1,     /* bad argument or size beyond a stated limit */
    LIMA_ERR_CUDA = 2,         /* a CUDA call failed; lima_last_error has the text */
    LIMA_ERR_CAPACITY = 3,     /* a neighbour list overflowed its capacity (reference: exit(1), Bodies.cuh:215-245) */
    LIMA_ERR_STATE = 4,        /* call out of order (e.g. step before lima_finish_box) */
    LIMA_ERR_NUMERIC = 5,      /* NaN position or |F| > 2e12 (reference: critical_error_encountered, Engine.cu:1050,1151) */
    LIMA_ERR_UNSUPPORTED = 6   /* feature not available in the selected semantics */
} lima_status;

typedef enum {
    /* The reference's own functional forms, list radii and integrator:
       LJ over entity neighbour lists with no force cutoff and per-path mixing
       rules, reference bonded forms, Stormer-Verlet with the reference
       thermostat scalar (Engine.cu:461-1223). */
    LIMA_SEMANTICS_REFERENCE = 0,
    /* Conservative physics of the same model: Lorentz-Berthelot LJ with a
       cutoff (+ optional potential switch) over a Verlet-buffered list,
       harmonic bonds/angles and periodic dihedrals as gradients of their
       energies, velocity Verlet, optional Berendsen thermostat. */
    LIMA_SEMANTICS_PHYSICS = 1
} lima_semantics;

typedef enum {
    LIMA_PRECISION_FP32 = 0,   /* plain FP32 state, forces and sums */
    LIMA_PRECISION_MIXED = 1   /* FP32 forces, compensated FP32 accumulation and state updates,
                                  FP64 energy/virial/KE reductions and thermostat scalar */
} lima_precision;

typedef enum {
    LIMA_THERMOSTAT_NONE = 0,
    LIMA_THERMOSTAT_REFERENCE = 1,  /* Engine::handleBoxtemp (Engine.cu:314-393): lambda = clamp(T0/T, 0.9, 1.1)
                                       applied to the position delta for one step every thermostat_period steps */
    LIMA_THERMOSTAT_BERENDSEN = 2   /* lambda = sqrt(1 + dt/tau (T0/T - 1)) on velocities every step */
} lima_thermostat;

typedef struct {
    float box_len;             /* nm, cubic periodic box (reference BOX_LEN, Constants.cuh:35) */
    float cutoff;              /* nm, physics cutoff r_c */
    float ref_cutoff;          /* nm, the reference's CUTOFF constant (Constants.cuh:52); lists use 2*ref_cutoff.
                                  0 = cutoff/2, so both semantics see the same list radius */
    float skin;                /* nm, Verlet buffer of the physics list */
    float switch_on;           /* nm, start of the C2 potential switch S = t^3 (10 - 15 t + 6 t^2),
                                  t = (cutoff^2 - r^2) / (cutoff^2 - switch_on^2) (physics); >= cutoff: plain shifted cutoff */
    double dt;                 /* ns */
    int nlist_period;          /* steps between list rebuilds (reference: 200, Constants.cuh:71); physics
                                  semantics: <= 0 rebuilds when a particle has moved more than skin/2
                                  (decided on the device), > 0 rebuilds every nlist_period steps and
                                  reports a list gone stale in between as LIMA_ERR_NUMERIC */
    int semantics;             /* lima_semantics */
    int precision;             /* lima_precision */
    int thermostat;            /* lima_thermostat */
    double t_target;           /* K */
    double tau_t;              /* ns, Berendsen coupling time */
    int thermostat_period;     /* steps, reference thermostat (Constants.cuh:82) */
    int energy_period;         /* steps between FP64 energy/virial evaluations (0 = only on lima_compute_energies) */
    int solvent_list_capacity; /* per-solvent solvent-neighbour capacity, reference semantics (power of two) */
    int compound_list_capacity;/* per-compound solvent-neighbour capacity, reference semantics */
    int device;                /* CUDA device ordinal */
    void* stream;              /* cudaStream_t to run on, or NULL for a library-owned stream */
} lima_params;

typedef struct lima_ctx lima_ctx;

/* Energies, FP64, of the last evaluated step (lima_get_energies totals[]). */
enum {
    LIMA_E_LJ = 0, LIMA_E_BOND = 1, LIMA_E_ANGLE = 2, LIMA_E_DIHEDRAL = 3,
    LIMA_E_KINETIC = 4, LIMA_E_VIRIAL = 5, LIMA_E_TEMPERATURE = 6, LIMA_E_TOTAL = 7,
    LIMA_E_COUNT = 8
};

/* Neighbour-list selectors for lima_get_nlist / lima_set_nlist. */
enum {
    LIMA_NL_COMPOUND_COMPOUND = 0,  /* NeighborList::neighborcompound_ids of compounds */
    LIMA_NL_COMPOUND_SOLVENT = 1,   /* NeighborList::neighborsolvent_ids of compounds */
    LIMA_NL_SOLVENT_COMPOUND = 2,   /* NeighborList::neighborcompound_ids of solvents */
    LIMA_NL_SOLVENT_SOLVENT = 3,    /* NeighborList::neighborsolvent_ids of solvents */
    LIMA_NL_PAIR = 4                /* physics semantics: the Verlet list of every particle */
};

/* Defaults: reference semantics, FP32, box 7 nm, cutoff 1.4 nm (reference
   CUTOFF 0.7), dt 1e-7 ns, list period 200, no thermostat. */
void lima_default_params(lima_params* p);

/* Replaces Engine::Engine(Simulation*, ForceField) (Engine.cu:9-38) together
   with lima_set_forcefield / lima_load_* / lima_finish_box. */
lima_status lima_create(const lima_params* params, lima_ctx** out);
void lima_destroy(lima_ctx* ctx);
const char* lima_last_error(const lima_ctx* ctx);

/* ForceField copy to the device (Engine.cu:27: cudaMemcpyToSymbol). */
lima_status lima_set_forcefield(lima_ctx* ctx, const lima_forcefield* ff);

/* Box contents (BoxBuilder::finishBox + Box::moveToDevice, BoxBuilder.cu:73-145,
   Simulation.cuh:73-91).  The caller keeps ownership of the host arrays. */
lima_status lima_load_compounds(lima_ctx* ctx, const lima_compound* compounds,
                                const lima_compound_state* states, int n_compounds);
lima_status lima_load_bridges(lima_ctx* ctx, const lima_compound_bridge_compact* bridges, int n_bridges);
lima_status lima_load_solvents(lima_ctx* ctx, const lima_solvent* solvents, uint32_t n_solvents);

/* Uploads the box and builds the first neighbour lists synchronously
   (Engine.cu:35: handleNLISTS(simulation, false, true)). */
lima_status lima_finish_box(lima_ctx* ctx);

/* n_steps of Engine::deviceMaster + Engine::hostMaster (Engine.cu:44-75,
   400-451): forces, integration, list rebuilds every nlist_period steps and
   the thermostat, all on the device with no host synchronisation inside. */
lima_status lima_step(lima_ctx* ctx, int n_steps);

/* Blocks until the engine's stream is idle and reports a device-side error
   (capacity overflow, NaN) raised since the last call. */
lima_status lima_synchronize(lima_ctx* ctx);

/* State readback in the reference layout (Box::compound_state_array,
   Compound::prev_positions, Box::solvents); compound slots past a compound's
   n_particles are zero in both arrays.  Either compound array may be NULL. */
lima_status lima_get_compound_states(lima_ctx* ctx, lima_compound_state* states, lima_float3* prev_positions);
lima_status lima_get_solvents(lima_ctx* ctx, lima_solvent* solvents);
/* The same positions as flat float arrays, for callers that do not use the
   reference's structs: compound particle (c, l) at compound_xyz[3 * (c * 64 + l)]
   (slots past a compound's n_particles are zero), solvent s at
   solvent_xyz[3 * s].  Either pointer may be NULL.  The reference's caller reads
   the same values from Box::compound_state_array and Box::solvents
   (Simulation.cuh:35-92). */
lima_status lima_get_positions(lima_ctx* ctx, float* compound_xyz, float* solvent_xyz);
/* Replace the positions of a loaded box in place (same layout as loading). */
lima_status lima_set_state(lima_ctx* ctx, const lima_compound_state* states, const lima_float3* prev_positions,
                           const lima_solvent* solvents);

/* Total force each particle was integrated with in the last step:
   compound_forces[c*64 + l], solvent_forces[s]. */
lima_status lima_get_forces(lima_ctx* ctx, lima_float3* compound_forces, lima_float3* solvent_forces);

/* FP64 energies (LIMA_E_*) and, optionally, the per-particle potE of the last
   step in the reference's potE_buffer indexing (compound c particle l at
   c*64+l, solvent s at n_compounds*64+s; Engine.cu:1012,1141). */
lima_status lima_get_energies(lima_ctx* ctx, double* totals, double* potE_per_particle);
/* Evaluates energies for the current positions without stepping. */
lima_status lima_compute_energies(lima_ctx* ctx);

/* Neighbour lists (Engine::updateNeighborLists, Engine.cu:208-287).
   lima_build_nlist runs one update now.  lima_get_nlist writes CSR offsets
   (n_entities+1) and ids (sorted ascending within each list); with ids NULL
   only offsets and *total are written.  lima_set_nlist installs a previous
   compound-compound list state, which the reference's update depends on.
   Physics semantics: LIMA_NL_PAIR gives the Verlet list of the last build,
   rows and ids in particle order (compound particles compound by compound,
   then solvents); the other selectors belong to reference semantics. */
lima_status lima_build_nlist(lima_ctx* ctx);
lima_status lima_get_nlist(lima_ctx* ctx, int which, uint32_t* offsets, uint32_t* ids, uint32_t* total);
lima_status lima_set_nlist(lima_ctx* ctx, int which, const uint32_t* offsets, const uint32_t* ids);

/* Physics semantics: pair-list builds since lima_finish_box (those at creation,
   lima_set_state and lima_build_nlist included).  With nlist_period <= 0 the
   list is rebuilt whenever a particle has moved more than skin/2 since the
   last build, decided on the device inside the step graph. */
lima_status lima_get_rebuild_count(lima_ctx* ctx, uint64_t* count);

/* Reference thermostat scalar for the next step (Box::thermostat_scalar,
   Simulation.cuh:70); 1 after it has been applied once. */
lima_status lima_set_thermostat_scalar(lima_ctx* ctx, float scalar);

lima_status lima_get_step(lima_ctx* ctx, uint64_t* step);

/* Device time of the last lima_step call, ms (CUDA events on the engine's
   stream) — the reference's Engine::timings (Engine.cu:448-450). */
lima_status lima_get_last_step_ms(lima_ctx* ctx, float* ms);

/* Per-kernel device time: runs n_steps (no graph) with CUDA events around
   each kernel group on the engine's stream and writes the mean ms per step
   into ms[LIMA_PROF_COUNT].  Groups: physics — neighbour rebuild (sort,
   permute, list), bonded terms, pair+integrate; reference — rebuild,
   bridges, compound<-solvent chunks + compound kernel, solvent kernel.
   The reference's Engine::timings splits force/copy/list time
   (Engine.cu:49-75, 400-451). */
enum { LIMA_PROF_TOTAL = 0, LIMA_PROF_NLIST = 1, LIMA_PROF_BONDED = 2, LIMA_PROF_PAIR = 3, LIMA_PROF_COMPOUND = 4,
       LIMA_PROF_COUNT = 5 };
lima_status lima_profile_steps(lima_ctx* ctx, int n_steps, float* ms);

/* Number of kernels of this library the context has launched so far
   (graph replays count the kernels they contain). */
lima_status lima_get_kernel_launches(lima_ctx* ctx, uint64_t* count);

/* ------------------------------------------------------------------ */
/* Parameter gradients of a trajectory loss (physics semantics).  The   */
/* reference has no gradients: LIMA_NET learns from trajectories the    */
/* engine writes (Environment.cpp:138-141).  Here the loss is           */
/* differentiated through the unrolled steps by a hand-written adjoint. */
/* ------------------------------------------------------------------ */
#define LIMA_LOSS_MAX_BINS 128

/* Parameter vector theta, n = 2 * n_types + 3 + 2 * (n_bond_types + n_angle_types +
   n_dihedral_types) entries:
     [sigma_0 .. sigma_{n_types-1}, epsilon_0 .. epsilon_{n_types-1},
      s_bond, s_angle, s_dihedral,
      (r0, k) of every bond type, (theta0, k) of every angle type, (phi0, k) of every dihedral type]
   n_types = 1 + the largest atom type in the box, sigma in nm and epsilon in J/mol
   (Lorentz-Berthelot mixing per pair).  A bonded term type is one distinct constant set
   among the loaded terms of a kind (PairBond {b0, kb}, AngleBond {theta_0, k_theta},
   DihedralBond {phi_0, k_phi, n}: Bodies.cuh:61-113), the types in ascending order of
   (r0, k), (theta0, k), (phi0, k, n); every term of a type takes its r0 / theta0 / phi0,
   and s_kind times its k as force constant (s_* = 1 as loaded).  The dihedral
   multiplicity n is an integer and not a parameter. */
lima_status lima_get_param_count(lima_ctx* ctx, int* n);
/* counts[4] = {n_types, n_bond_types, n_angle_types, n_dihedral_types}. */
lima_status lima_get_param_layout(lima_ctx* ctx, int* counts);
/* The number of terms of a kind (0 bond, 1 angle, 2 dihedral) and, when type_of is not
   NULL, the type of each, in load order: each compound's terms compound by compound,
   then each bridge's terms. */
lima_status lima_get_bonded_types(lima_ctx* ctx, int kind, int* n_terms, int* type_of);
lima_status lima_get_params(lima_ctx* ctx, double* theta);
lima_status lima_set_params(lima_ctx* ctx, const double* theta);

typedef struct {
    int n_steps;             /* T: the loss averages over the states after steps 1..T */
    int checkpoint_every;    /* C: the forward pass keeps every C-th state and the backward pass
                                recomputes each C-step segment from it (C >= T: one segment) */
    int n_bins;              /* RDF bins, 1..LIMA_LOSS_MAX_BINS */
    float r_max;             /* nm: bins of width dr = r_max / n_bins over [0, r_max];
                                r_max + dr <= cutoff (the B-spline support) */
    double w_energy;         /* weight of the potential energy per particle, U / N (J/mol) */
    double w_rdf;            /* weight of the RDF-bin term */
    const double* rdf_target;/* n_bins target occupancies (host); may be NULL when w_rdf == 0 */
} lima_loss_spec;

/* loss = (1/T) sum_{n=1..T} [ w_energy U(x_n)/N + w_rdf sum_b (h_b(x_n) - target_b)^2 ] with
   h_b(x) = (1/N) sum over non-excluded pairs i<j of B(r_ij/dr - b - 1/2), B the quadratic
   B-spline (support |u| < 3/2; the bins of one distance sum to 1).  Both calls run T NVE
   velocity-Verlet steps of the physics path from the current state (plain FP32, thermostat
   none, potential switch on), re-sort and rebuild the pair list at every checkpoint and
   rebuild it in place every 10 steps in between (it must stay valid for 10 steps:
   LIMA_ERR_NUMERIC otherwise), and leave the state as they found it. */
lima_status lima_loss(lima_ctx* ctx, const lima_loss_spec* spec, double* loss);
/* The same loss and d loss / d theta (lima_get_params order), by the adjoint of the unrolled
   steps: pair and bonded Hessian-vector products in FP32, FP64 parameter reductions. */
lima_status lima_grad(lima_ctx* ctx, const lima_loss_spec* spec, double* loss, double* grad);
/* h_b of the current state (definition above), e.g. to build a target. */
lima_status lima_rdf(lima_ctx* ctx, int n_bins, float r_max, double* h);

/* ------------------------------------------------------------------ */
/* Frame log (either semantics).  Replaces the reference's logging      */
/* buffers written by the force kernels every step (Box::potE_buffer,   */
/* traj_buffer, outdata, data_GAN: Engine.cu:1007-1047, 1136-1145),      */
/* their host offload every 40 / 100 steps (Engine::hostMaster,          */
/* offloadLoggingData, offloadTrainData: Engine.cu:44-75, 290-310), the  */
/* post-run Analyzer::analyzeEnergy (Analyzer.cu:33-207) and the output  */
/* files of Environment::postRunEvents (Environment.cpp:124-166).        */
/* ------------------------------------------------------------------ */
#define LIMA_LOG_TRAJ 1     /* positions of every particle slot (traj_buffer) */
#define LIMA_LOG_POTE 2     /* potential energy of every particle slot (potE_buffer): its LJ pair halves
                               plus 1/2, 1/3, 1/4 of each bond, angle, dihedral it takes part in */
#define LIMA_LOG_TRAIN 4    /* compound particles: position, LJ force from solvents, 0 (data_GAN,
                               N_DATAGAN_VALUES = 3 float3; padding particles at (-1, -1, -1)) */
#define LIMA_LOG_DATA_FLOATS 10   /* outdata floats per frame (Engine.cu:1022-1029) */

typedef struct {
    int every;          /* record the state of every `every`-th step (step % every == 0), >= 1;
                           the reference records every step */
    int ring_frames;    /* frames held in device memory between copies to the host, 1..65536 */
    int flags;          /* LIMA_LOG_* (the FP64 energies and the outdata line are always recorded) */
} lima_log_params;

/* Starts recording (clears what an earlier start recorded).  A recorded step
   runs the step's energy variant.  Frame f of step s holds the positions the
   step's forces were evaluated at, that evaluation's energies, and the
   velocity of the half step taken.  Layout per frame: traj[n_slots][3] float,
   potE[n_slots] double, n_slots = n_compounds*64 + n_solvents (compound c
   particle l at c*64 + l, solvent s at n_compounds*64 + s; empty compound
   slots are zero); train[n_compounds*64][3][3] float; energies[LIMA_E_COUNT]
   double; logdata[10] float (particle slot 0: speed, kinetic energy,
   potential energy, |force|, then zeros).
   Reference semantics records what the reference's step writes instead: the
   positions after the step, the compound particles' potE of the step's
   compound kernel (solvent slots 0), data_GAN (position or (-1, -1, -1), then
   force_LJ_sol), the outdata line of compound 0 particle 0 and, as energies,
   the bonded potE summed over the compound slots and the last thermostat
   temperature; energy.bin then holds the Analyzer's central-difference
   energies of frames 1 .. F-3, over frames `every` steps apart (the
   reference records every step). */
lima_status lima_log_start(lima_ctx* ctx, const lima_log_params* params);
/* Stops recording; what was recorded stays readable. */
lima_status lima_log_stop(lima_ctx* ctx);
/* Frames recorded so far (waits for the engine's stream). */
lima_status lima_log_count(lima_ctx* ctx, uint64_t* n_frames);
/* Frames [first, first+count) into caller arrays (any may be NULL; traj,
   potE and train need the matching flag). */
lima_status lima_log_read(lima_ctx* ctx, uint64_t first, uint64_t count, uint64_t* steps, double* energies,
                          float* traj, double* potE, float* train, float* logdata);
/* The recorded frames as the reference's output files in directory `dir`
   (which must exist): logdata.bin (10 float per frame), energy.bin (float3
   per frame: potential, kinetic and total energy per particle, J/mol),
   temperature.bin (float per frame, K), sim_traindata.bin (with
   LIMA_LOG_TRAIN: 3 float3 per compound particle slot per frame); with
   LIMA_LOG_TRAJ / LIMA_LOG_POTE also traj.bin (float3 per slot per frame)
   and potE.bin (double per slot per frame), the in-memory
   Simulation::traj_buffer / potE_buffer of the reference. */
lima_status lima_log_write(lima_ctx* ctx, const char* dir);

/* ------------------------------------------------------------------ */
/* Headless rasterizer.  Replaces Rasterizer::render (Rasterizer.cu:     */
/* 12-294) and the picture DisplayV2::drawBalls draws from its output    */
/* (DisplayV2.cpp:13-51); there is no window or OpenGL context.          */
/* ------------------------------------------------------------------ */
typedef struct {
    lima_float3 pos;      /* normalised: (x / box_len - 0.5) * 1.8 per axis; drawn at (pos.x, pos.z) */
    float radius;         /* 0.25 * r_type / (1 + 0.001 * y_nm) */
    int32_t color[3];     /* RGB 0..255 of the atom type */
    uint8_t disable;      /* 1 for an empty compound slot */
    uint8_t pad[3];
} lima_render_ball;       /* RenderBall (QuantomTypes.cuh:362-369), 32 bytes */

/* One ball per particle slot (n_compounds*64 + n_solvents, compound c
   particle l at c*64 + l, solvents after) of the current state, sorted by
   pos.y ascending (ties in slot order).  Atom types: compound particles from
   atom_color_types (0 SOL, 1 C, 2 O, 3 N, 4 H, 5 P, 6 SOL, else NONE),
   solvents SOL, empty slots NONE at the box origin, disabled. */
lima_status lima_render(lima_ctx* ctx, lima_render_ball* balls);
/* The same balls drawn as the reference's display draws them, into a
   width x height RGB image (row 0 at the top, device coordinates [-1, 1]
   on both axes, black background): every pixel whose centre lies in a ball's
   disc takes the colour of the front-most such ball (lowest pos.y), scaled by
   the Gouraud light of the display's triangle fan, 0.5 + 0.5 * dy / radius
   (floor per channel).  width, height 1..16384. */
lima_status lima_render_image(lima_ctx* ctx, int width, int height, uint8_t* rgb);

/* ------------------------------------------------------------------ */
/* Real-topology input.  Replaces the reference's input path:           */
/* LIMA_ForcefieldMaker (CHARMM parameter files -> typed tables,         */
/* LIMA_ForcefieldMaker.cpp:16-146), ForceFieldMaker::buildForcefield    */
/* (Forcefield.cu:10-218), CompoundBuilder::buildMolecule                 */
/* (CompoundBuilder.cpp:7-463) and BoxBuilder::addSingleMolecule /       */
/* solvateBox (BoxBuilder.cu:42-218), as in Environment::Environment     */
/* (Environment.cpp:15-40).  The result is the box arrays lima_load_*    */
/* take.                                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    float box_len;        /* nm; the molecule's centre goes to the box centre (BOX_LEN, Constants.cuh:35) */
    int min_residue_id;   /* residues before min_residue_id are skipped, reading stops after max_residue_id */
    int max_residue_id;
    int ignore_hydrogens; /* 1: atoms whose name starts with 'H' and every term touching them are left out */
    int solvate;          /* 1: the conf's SOL oxygens become solvents where no compound particle is within
                             0.2 nm and no earlier solvent within 0.25 nm (BoxBuilder.cu:194-218, 440-461) */
    double dt;            /* ns; a solvent's previous position is pos - v dt */
    double temperature;   /* K; solvent speed sqrt(3 R T / M) (BoxBuilder.cuh:63-71) */
    uint64_t seed;        /* solvent velocity directions (uniform on the sphere) */
} lima_topology_options;

typedef struct lima_topology lima_topology;

/* Defaults of the reference's demo (Environment.cpp:21-24, Constants.cuh:35,
   Simulation.cuh:152): 7 nm box, residues 0..200, hydrogens left out,
   solvated, dt 1e-7 ns, 313 K. */
void lima_topology_default_options(lima_topology_options* options);
/* Builds the box from a GROMACS conf.gro, its topol.top and CHARMM parameter
   files (read in the order given).  *out is set even on failure (then
   lima_topology_error says why); free it with lima_topology_destroy. */
lima_status lima_topology_build(const char* gro_path, const char* top_path, const char* const* prm_paths, int n_prm,
                                const lima_topology_options* options, lima_topology** out);
const char* lima_topology_error(const lima_topology* topology);
lima_status lima_topology_sizes(const lima_topology* topology, int* n_compounds, int* n_bridges, uint32_t* n_solvents,
                                int* n_atom_types);
/* Copies the box into caller arrays sized by lima_topology_sizes (any may be NULL). */
lima_status lima_topology_export(const lima_topology* topology, lima_forcefield* forcefield, lima_compound* compounds,
                                 lima_compound_state* states, lima_compound_bridge_compact* bridges,
                                 lima_solvent* solvents);
void lima_topology_destroy(lima_topology* topology);

/* ------------------------------------------------------------------ */
/* No counterpart in the reference.  The reference updates its lists on  */
/* the host (Engine::updateNeighborLists, Engine.cu:208-287); this is a  */
/* context-free, allocation-free form of the device build behind          */
/* lima_build_nlist for the solvent-solvent list.                         */
/* ------------------------------------------------------------------ */
#define LIMA_NOALLOC_MAX_SOLVENTS 65536

/* Solvent-solvent neighbour list of the reference semantics,
   {i<j : within(pos_i, pos_j, cutoff + cutoff)} mirrored to both rows and
   sorted ascending.  This is what lima_get_nlist(LIMA_NL_SOLVENT_SOLVENT)
   returns after lima_build_nlist. It is built on caller-owned device buffers
   and allocates no memory.  It is for callers that cannot allocate device
   memory: memory reserved up front, or a loop that must not call
   cudaMalloc/cudaFree, which can wait on other streams' work.  Such callers
   cannot use lima_ctx, whose buffers lima_finish_box allocates.  The cell grid
   and staged positions live in one fixed 1,966,080-byte device array of the
   library.  Hence the limits:
     n_solvents 1..LIMA_NOALLOC_MAX_SOLVENTS; capacity 32..2048
     (LIMA_ERR_CAPACITY beyond either).
   Buffers (device memory of the current device):
     d_solvents  n_solvents reference Solvent records (only pos is read);
     d_ids       capacity * n_solvents; entry k of solvent i at d_ids[k * n_solvents + i];
     d_counts    n_solvents row lengths, clamped to capacity;
     d_overflow  one int: zeroed by the call; nonzero once the work has run if
                 a row held more than capacity neighbours.
   cutoff is the reference CUTOFF (list radius 2 * cutoff).  The work is queued
   on `stream` (a cudaStream_t; NULL is the default stream) and the call returns
   without waiting.  The first call on a device looks up the array's address
   there (cudaGetSymbolAddress), so make it before any stream capture on that
   device.  The address is kept per device ordinal for the rest of the process:
   it belongs to the device's primary context, so call this with the primary
   context current, and not after cudaDeviceReset (which ends that context).
   Every call on a device shares the one array: calls that overlap in time,
   from other streams or host threads, race.  err (may be NULL) receives a
   message on failure. */
lima_status lima_ss_nlist_noalloc(const lima_solvent* d_solvents, int n_solvents, float box_len, float cutoff,
                                  int capacity, uint32_t* d_ids, uint32_t* d_counts, int* d_overflow, void* stream,
                                  char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* LIMA_ABI_H */
