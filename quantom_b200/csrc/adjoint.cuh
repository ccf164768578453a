// Parameter gradients of a trajectory loss on the physics path: the adjoint
// of the unrolled velocity-Verlet steps with checkpointed recomputation.
//
// Step n -> n+1 (NVE, kick-drift form, F = -grad U):
//   v_{n+1/2} = v_{n-1/2} + dt F(x_n) / m,   x_{n+1} = x_n + dt v_{n+1/2}
// Backward, with lx = dL/dx_{n+1} and lv = dL/dv_{n+1/2}:
//   mu = lv + dt lx;  w = mu / m
//   dL/dv_{n-1/2} = mu
//   dL/dx_n = lx + dt (dF/dx)(x_n) w + dl_n/dx_n          ((dF/dx) is symmetric)
//   dL/dtheta += dt sum_i w_i . dF_i/dtheta (x_n) + dl_n/dtheta
// The force Jacobian is applied per pair (analytic d f / d r^2 of the
// switched LJ force) and per bonded term (forward-mode dual numbers).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lima_abi.h"
#include "physdev.cuh"

namespace lima {

// parameter slots after the per-type sigma / epsilon entries
enum { kParBond = 0, kParAngle = 1, kParDihedral = 2, kParKinds = 3 };

// Host copy of the differentiable parameters and of the bonded constants as loaded.
// A bonded term type is one distinct constant set among the loaded terms of a
// kind: (r0, k) of a bond, (theta0, k) of an angle, (phi0, k, n) of a
// dihedral, in ascending order of that tuple.  The reference's force field
// gives every term of one atom-type combination the same constants
// (Bodies.cuh:61-113, filled per type by its force-field maker), so the
// distinct sets are its bond / angle / dihedral types.
struct PhysParams {
    int n_types = 0;
    std::vector<double> sigma, epsilon;      // per type
    double scale[kParKinds] = {1.0, 1.0, 1.0};
    std::vector<float2> bond0, angle0;       // (r0, k), (theta0, k) as loaded
    std::vector<float4> dih0;                // (phi0, k, n, 0) as loaded
    std::vector<int> type_of[kParKinds];     // term -> its type, per kind
    std::vector<float4> type0[kParKinds];    // the type's constants as loaded (c, k, n, 0)
    std::vector<double> tc[kParKinds], tk[kParKinds];   // current c (r0 / theta0 / phi0) and k per type
    int n_term_types() const {
        return (int)(type0[kParBond].size() + type0[kParAngle].size() + type0[kParDihedral].size());
    }
    int count() const { return 2 * n_types + kParKinds + 2 * n_term_types(); }
};

// Device buffers of the loss / adjoint passes (grown on demand).
struct AdjBuffers {
    int cap_ckpt = 0, cap_seg = 0, cap_steps = 0, cap_bins = 0;
    float4* ck_x = nullptr;   // [cap_ckpt][n]  checkpoint positions (w = type), orig order
    float4* ck_v = nullptr;   // [cap_ckpt][n]  checkpoint half-step velocities (w = 1/m)
    float4* seg_x = nullptr;  // [cap_seg][n_pad] positions of a recomputed segment, sorted order
    float4* seg_xo = nullptr; // [cap_seg][n_cp]  compound positions of those states, orig order
    float4* lam_x = nullptr;  // [n_pad] dL/dx, sorted order
    float4* lam_v = nullptr;  // [n_pad] dL/dv, sorted order
    float4* wv = nullptr;     // [n_pad] mu / m, sorted order
    float4* lam_xo = nullptr; // [n] dL/dx between segments, orig order
    float4* lam_vo = nullptr; // [n]
    float4* adj_term = nullptr;   // [n_term_slots] per (bonded term, atom) adjoint contribution
    double* U = nullptr;      // [cap_steps + 1] potential energy of state n
    double* hist = nullptr;   // [(cap_steps + 1) * cap_bins] h_b of state n
    double* target = nullptr; // [cap_bins]
    double* gtheta = nullptr; // [2 * kMaxTypes + kParKinds]
    float* par = nullptr;     // [2 * kMaxTypes + kParKinds] current theta (float)
    double2* gterm = nullptr; // [cap_terms] per bonded term: dL/d(r0 | theta0 | phi0), dL/dk of the term
    int cap_terms = 0;
};

void phys_params_init(const PhysDev& d, const lima_forcefield& ff, PhysParams& pp, cudaStream_t s);
// theta layout (PhysParams::count() entries): sigma[n_types], epsilon[n_types],
// s_bond, s_angle, s_dihedral, then (r0, k) per bond type, (theta0, k) per
// angle type, (phi0, k) per dihedral type; a term's force constant is
// s_kind * k of its type.  phys_params_set uploads theta into the LJ table and
// the bonded constants and returns a lima_status.
int phys_params_set(PhysDev& d, PhysParams& pp, const double* theta, std::string& msg, cudaStream_t s);
void phys_params_get(const PhysParams& pp, double* theta);

// Loss (and, with grad != nullptr, its gradient) of spec over the unrolled
// steps from the state in parity `cur`; the state is restored afterwards.
// Returns a lima_status; device buffers are appended to `allocs`.
int adj_run(const PhysDev& d, int cur, const PhysParams& pp, AdjBuffers& A, std::vector<void*>& allocs,
            const lima_loss_spec& spec, double* loss, double* grad, cudaStream_t s, std::string& msg);
// h_b of the state in parity `cur`
int adj_rdf(const PhysDev& d, int cur, AdjBuffers& A, std::vector<void*>& allocs, int n_bins, float r_max,
            double* h, cudaStream_t s, std::string& msg);

}  // namespace lima
