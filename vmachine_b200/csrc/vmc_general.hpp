// General walker path (vmc_general.cu): FP64 kernels for every wave-function
// element, used when a system has SimpleJastrow, RBM or hydrogen-orbital parts, and an
// FP32 sweep of the compiled atom form for mixed precision.
#pragma once
#include <string>

#include "vmc_config.hpp"
#include "vmc_kernels.cuh"

namespace vmc {

enum : int { BASIS_HERMITE = 1, BASIS_HYDROGEN = 2 };
// GEN_INIT: fresh walkers (masks, inverse, evaluation, force cache); GEN_STATE:
// evaluation; GEN_REFRESH: FP64 re-inversion from the positions and evaluation (the
// refresh of the atoms' FP32 sweep)
enum : int { GEN_INIT = 0, GEN_STATE = 1, GEN_REFRESH = 2 };
// Compiled variants of the general path: GV_ANY takes every element, basis and
// dimension at run time; GV_ATOM is the atoms' form (3D, a Slater determinant of
// hydrogen orbitals with SimpleJastrow and/or Pade-Jastrow) with the dimension and the
// element set compiled in, so per-coordinate arrays stay in registers and the
// sweep's code is a fraction of the generic one.
enum : int { GV_ANY = 0, GV_ATOM = 1 };
__host__ __device__ constexpr int gv_dim(int gv, int dim) { return gv == GV_ATOM ? 3 : dim; }
__host__ __device__ constexpr bool gv_has(int gv, int kind) { return gv == GV_ANY || (kind >= 1 && kind <= 3); }

// Record layout (offsets in doubles), element data and orbital table of the
// general path; passed by value to its kernels.
struct GenParams {
    int D, n, EP, p_max;        // coordinates, orbitals per block, E x p_max, p_max
    int off_fc, off_g, off_en, off_pg, off_inv, rec;
    int basis, hidden;          // BASIS_*, RBMProduct hidden units
    int horb3;                  // n = 3 hydrogen orbitals with the reference's second derivatives
    double sigma;               // RBM width
    const double *theta;        // E x p_max parameters on the device
    const float *mlp;           // MLP Jastrow weights rounded to bfloat16 (MLP_PARAMS), or null
    int off_uc, off_oc;         // MLP caches: (u, u', u'') per pair i < j, (chi, chi', chi'') per particle
    int off_dphi;               // Slater: d phi_o / dx_c and d2 phi_o / dx_c^2 at particle q, [q][o][2 dim]
    // parameters accumulated per walker (all but padding and the MLP row, whose
    // gradient comes from snapshots): accumulator 9 + c holds parameter act[c]
    const int *act;
    int n_act;
    int mlp_tc;                 // MLP sweep with the second layer on the tensor cores
    int variant;                // GV_*: the compiled sweep that takes this system
    int seg;                    // walkers per warp of the sweep (4: atoms of at most 4 electrons)
    int f32;                    // the sweep in FP32 (mixed precision, compiled atom form only)
    unsigned char orb[32][3];   // Hermite degrees (m0, m1, m2) or hydrogen (n, l, m + 1)
};


// "" when the general path takes the configuration (fills g except theta), else why not.
std::string gen_configure(const Config &c, int n_elements, int p_max, GenParams &g);
// Initialise (invert the Slater blocks, evaluate, force cache) or re-evaluate every
// walker; with output pointers, also the per-element values of vmc_eval.
cudaError_t gen_launch_state(const Params &P, const GenParams &g, int mode, double *o_grad, double *o_lap,
                             double *o_pg, double *o_en, cudaStream_t st);
cudaError_t gen_launch_sweep(const SweepArgs &a, const GenParams &g, cudaStream_t st);
cudaError_t upload_hermite_gen(const HermiteCoef &h);
// dJ/dtheta of the MLP Jastrow summed over snapshots (positions n_snap x D floats,
// local energies n_snap, or null = weights 0): out[0..P) += sum dJ/dtheta,
// out[P..2P) += sum E dJ/dtheta (FP64 accumulators, zeroed by the caller).  With
// g.mlp_tc and a fail word, the pair network's products run on the tensor cores and
// a completion wait that gives up ORs ST_TC_TIMEOUT into *fail.
cudaError_t mlp_launch_grad(const GenParams &g, int N, int dim, const float *snap_x, const double *snap_e,
                            long long n_snap, double *out, cudaStream_t st, unsigned *fail = nullptr);

}  // namespace vmc
