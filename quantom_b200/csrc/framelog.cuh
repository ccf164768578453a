// Frame log: the reference's on-device logging buffers
// (Box::potE_buffer / traj_buffer / outdata / data_GAN, Engine.cu:1007-1047
// and :1136-1145), its host offload (Engine::offloadLoggingData /
// offloadTrainData, Engine.cu:290-310) and the per-step energies of its
// post-run Analyzer (Analyzer.cu:33-207), recorded every `every` steps.
//
// A logged step is the step's energy variant (FP64 LJ / bonded / kinetic /
// virial reductions) followed by k_log_frame, which writes frame r of a
// device ring in the reference's particle indexing (compound c particle l at
// c*64 + l, solvent s at n_c*64 + s), and, for the train data, k_log_train.
// When the ring is full it is copied, stream-ordered, into one of two pinned
// host buffers (the next kernels that overwrite the ring come after the copy
// on the same stream), and the host moves that buffer into its store the
// next time it needs it.  No step waits for the host unless the host falls
// two rings behind.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lima_abi.h"
#include "physdev.cuh"
#include "refdev.cuh"

namespace lima {

constexpr int kLogDataFloats = 10;      // Box::outdata floats per step (Engine.cu:1022-1029)
constexpr int kTrainValues = 3;         // N_DATAGAN_VALUES (Constants.cuh:98)

// device-side view of one ring
struct FrameLogDev {
    int flags;
    int n_slots;            // n_c * 64 + n_s
    int n_train;            // n_c * 64
    int ring;
    const uint32_t* ref_slot;   // [n] orig id -> reference slot
    float* traj;            // [ring][n_slots][3]
    double* potE;           // [ring][n_slots]
    float* train;           // [ring][n_train][3 values][3]
    double* energies;       // [ring][LIMA_E_COUNT]
    float* logdata;         // [ring][10]
    // physics: frames written to the ring since its last drain; the kernels of
    // a frame write at ring position frame_ctr % ring, and the last block of
    // k_log_frame advances it (so a captured step graph can log)
    unsigned long long* frame_ctr;
    unsigned int* blocks_done;
};

struct FrameLog {
    bool on = false;
    int every = 0;
    FrameLogDev dev{};
    std::vector<void*> dallocs;     // device buffers from the process's stream-ordered pool
    cudaStream_t stream = nullptr;  // the engine's stream (allocations, frees and copies)
    // pinned staging, two rings; pending[b] = frames copied into b not yet in the store
    void* pinned[2] = {nullptr, nullptr};
    size_t ring_bytes = 0;
    int pending[2] = {0, 0};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int next_buf = 0;
    int in_ring = 0;                 // frames written to the device ring since its last drain
    // host store (every frame since lima_log_start)
    std::vector<uint64_t> steps;
    std::vector<float> traj;
    std::vector<double> potE;
    std::vector<float> train;
    std::vector<double> energies;
    std::vector<float> logdata;
    uint64_t frames_logged = 0;      // frames launched (some may still be on the device)
    std::vector<uint64_t> ring_steps;   // steps of the frames in the device ring
    std::vector<uint64_t> buf_steps[2];
};

// sets up a ring for the loaded box: n_s solvents, n_compound_particles[c] per compound
void framelog_start(FrameLog& g, int n_s, const std::vector<int>& n_compound_particles, const lima_log_params& p,
                    cudaStream_t s, std::string& msg, int& status);
void framelog_free(FrameLog& g);
// after the energy variant of step `step` on parity `cur` (accumulator slot `cur`)
int framelog_record(FrameLog& g, const PhysDev& d, int cur, uint64_t step, cudaStream_t s);
// the two halves of framelog_record: the frame's kernels (stream-ordered, also
// inside a graph capture) and the host's record of the frame (ring position,
// drain when the ring is full)
int framelog_launch(const FrameLog& g, const PhysDev& d, int cur, cudaStream_t s);
void framelog_note(FrameLog& g, uint64_t step, cudaStream_t s);
// reference semantics: after step `step`, whose positions are in parity `after`
int framelog_record_ref(FrameLog& g, const RefDev& d, int after, uint64_t step, cudaStream_t s);
// every frame launched so far into the host store (waits for the stream)
void framelog_flush(FrameLog& g, cudaStream_t s);

}  // namespace lima
