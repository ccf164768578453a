// Replacement for the reference's compile-time configuration header
// (Quantom/Quantom/Constants.cuh:6-113), used only by the host build of the
// reference engine in oracle/_ref.  The build script copies the reference
// sources to a temporary directory and puts this file in place of the
// original, so that:
//  * BOX_LEN / BOX_LEN_HALF / CUTOFF become runtime globals (set through the
//    oracle's C API) instead of constexpr values — every benchmark box has
//    its own box length and cutoff;
//  * the neighbour-list capacities are raised so a host run never overflows
//    (NeighborList::addId calls exit(1) on overflow, Bodies.cuh:215-245);
//  * MAX_SOLVENTS is lowered from 0xFFFF to 32767 so the host-side
//    NListDataCollection (Engine.cuh:61-105) stays a few hundred MB.
// The feature switches keep the reference's settings.
#pragma once

#define LIMA_DEBUGMODE
#define ENABLE_SOLVENTS
#define ENABLE_BLJV
#define ENABLE_DIHEDRALS

const bool print_compound_positions = false;

extern float BOX_LEN;        // nm, runtime (reference: constexpr 7.f)
extern float BOX_LEN_HALF;   // nm, runtime, always BOX_LEN / 2
extern float CUTOFF;         // nm, runtime (reference: 0.7f)

const int N_SOLVATE_MOLECULES = 2000;

const int NEIGHBORLIST_MAX_COMPOUNDS = 64;
const int NEIGHBORLIST_MAX_SOLVENTS = 6144;   // reference: 1024
const int SOLVENTS_BATCHSIZE = 64;

const int MAX_SOLVENTS = 32767;               // reference: 0xFFFF

const int MAX_COMPOUND_PARTICLES = 64;
const int THREADS_PER_SOLVENTBLOCK = 128;
const int THREADS_PER_COMPOUNDBLOCK = MAX_COMPOUND_PARTICLES;

const int SIMULATION_STEPS = 100000;
const int STEPS_PER_NLIST_UPDATE = 200;
const int STEPS_PER_RENDER = 200;

const int STEPS_PER_LOGTRANSFER = 40;
const int STEPS_PER_THERMOSTAT = 40;
const bool ENABLE_BOXTEMP = true;
const bool APPLY_THERMOSTAT = true;
const bool PRINT_TEMP = false;

const int MAX_COMPOUNDS = 0xFF;
const int MAX_ATOMS = 1000000;
const int MAX_ATOMS_IN_RESIDUE = 32;

const int N_DATAGAN_VALUES = 3;
const int STEPS_PER_TRAINDATATRANSFER = 100;

const int COMPOUNDBRIDGES_IN_BUNDLE = 64;
const int MAX_PARTICLES_IN_BRIDGE = 32;
const int MAX_SINGLEBONDS_IN_BRIDGE = 32;
const int MAX_ANGLEBONDS_IN_BRIDGE = 32;
const int MAX_DIHEDRALBONDS_IN_BRIDGE = 32;
