// Test infrastructure (oracle): drives the reference's own input path
// (ForceFieldMaker, CompoundBuilder::buildMolecule, BoxBuilder as in
// Environment::Environment, Environment.cpp:15-40) on files already prepared
// by the reference's LIMA_ForcefieldMaker, and dumps the resulting box:
//   int32 n_compounds, n_bridges, n_solvents
//   ForceField (384 B), Compound[n_compounds], CompoundState[n_compounds],
//   CompoundBridgeCompact[n_bridges], Solvent[n_solvents]
// Built by oracle/build_ref_input.sh against a copy of the reference sources;
// never linked into the product.
#include "CompoundBuilder.h"
#include "BoxBuilder.cuh"

#include <cstdio>

[[noreturn]] void lima_ref_exit(int code) {
    std::fprintf(stderr, "reference input path exited with %d\n", code);
    (std::exit)(code ? code : 70);
}
thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
void __syncthreads() {}

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s out.bin (run from a directory whose ../../Simulation holds the inputs)\n", argv[0]);
        return 2;
    }
    Simulation* sim = new Simulation();
    ForceFieldMaker* ffm = new ForceFieldMaker();
    CompoundBuilder cb(ffm);
    Molecule mol = cb.buildMolecule(MOL_FOLDER + "conf.gro", MOL_FOLDER + "topol.top", 200, 0, true);
    std::vector<Float3> sol = cb.getSolventPositions(MOL_FOLDER + "conf.gro");
    BoxBuilder bb;
    bb.buildBox(sim);
    bb.addSingleMolecule(sim, &mol);
    bb.solvateBox(sim, &sol);
    Box* box = sim->box;
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 3;
    const int32_t counts[3] = {(int32_t)box->n_compounds, (int32_t)box->bridge_bundle->n_bridges,
                               (int32_t)box->n_solvents};
    ForceField ff = ffm->getNBForcefield();
    std::fwrite(counts, sizeof counts, 1, f);
    std::fwrite(&ff, sizeof ff, 1, f);
    std::fwrite(box->compounds, sizeof(Compound), box->n_compounds, f);
    std::fwrite(box->compound_state_array, sizeof(CompoundState), box->n_compounds, f);
    std::fwrite(box->bridge_bundle->compound_bridges, sizeof(CompoundBridgeCompact), box->bridge_bundle->n_bridges, f);
    std::fwrite(box->solvents, sizeof(Solvent), box->n_solvents, f);
    std::fclose(f);
    return 0;
}
