/* vmc_oracle — CPU restatement of VMaChine's hot path, in plain C (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load this library, and only as the checker.  The product
 * path (vmachine_b200) never links or calls it.
 *
 * It restates, function by function, the reference's algorithm (evenmn/VMaChine,
 * file:line cited beside each function in vmc_oracle.c) with one deliberate
 * difference in *how* it computes: every step re-evaluates the wave function from
 * the positions (fresh Gauss-Jordan inverse of each Slater block, full pair sums),
 * instead of carrying the reference's incremental arrays.  That makes it an
 * independent check of the GPU engine's incremental (Sherman-Morrison, running
 * pair sums) algorithm.  It is pinned against the compiled reference itself:
 * tests/golden/ holds vectors made by oracle/_ref (the reference's own sources),
 * and tests/test_oracle_pin.py checks this file against them.
 */
#ifndef VMC_ORACLE_H
#define VMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    VMO_GAUSSIAN = 0,
    VMO_SLATER = 1,
    VMO_PADE = 2,
    VMO_SIMPLEJASTROW = 3,
    VMO_RBMGAUSSIAN = 4,
    VMO_RBMPRODUCT = 5,
    VMO_HYDROGENLIKE = 6,
};
enum { VMO_BASIS_NONE = 0, VMO_BASIS_HERMITE = 1, VMO_BASIS_HYDROGEN = 2 };
enum { VMO_HAM_HO = 0, VMO_HAM_ATOM = 1 };
enum { VMO_IS = 0, VMO_BF = 1 };
/* compat flags: bit set = reproduce the reference quirk */
enum {
    VMO_Q_PADE_RATIO = 1,     /* Pade ratio over j >= moved particle only (padejastrow.cpp:214) */
    VMO_Q_PADE_DGAMMA = 2,    /* dlnPsi/dgamma halved (padejastrow.cpp:114)                     */
    VMO_Q_SJ_RATIO = 4,       /* SimpleJastrow ratio over j > moved particle only (simplejastrow.cpp:148) */
    VMO_Q_IS_GREEN = 8,       /* IS Green's ratio as in importancesampling.cpp:43-47,58          */
    VMO_Q_RBM_SORT = 16,      /* RBMProduct hidden units see sorted coordinates (wavefunction.cpp:40-55) */
    VMO_Q_HORB3 = 32,         /* n = 3 hydrogen-orbital second derivatives as hydrogenorbital.cpp:351-364 */
    VMO_Q_ALL = 63,
};

#define VMO_MAX_ELEM 8

typedef struct {
    int N, d;                 /* particles, dimensions */
    int n_elem;
    int elem[VMO_MAX_ELEM];   /* element codes, in configuration order */
    int basis;                /* VMO_BASIS_* */
    int hamiltonian;          /* VMO_HAM_* */
    int coulomb;              /* 1 = Coulomb interaction */
    int sampling;             /* VMO_IS / VMO_BF */
    int hidden;               /* RBM hidden nodes */
    int p_max;                /* parameters per element row */
    int quirks;               /* VMO_Q_* bits */
    double omega, Z, step;    /* omega, atomic number, stepLength (dt for IS) */
    double sigma;             /* RBM width (1/sqrt(omega) after the omega key) */
    double drift_limit;       /* corrected IS: drift limiter a (0: off), v -> 2v / (1 + sqrt(1 + 2 a dt v^2)) */
} vmo_system;

/* Per-element parameter count (the reference's getNumberOfParameters after setConstants). */
int vmo_num_parameters(const vmo_system *s, int element_index);

/* Evaluate at fixed positions.  theta: n_elem x p_max (row-major).
 * grad: n_elem x D, lap: n_elem, pgrad: n_elem x p_max, energies: {T, V_ext, V_int}.
 * Returns 0, or <0 for a singular Slater block. */
int vmo_eval(const vmo_system *s, const double *theta, const double *pos, double *grad,
             double *lap, double *pgrad, double *energies);

/* Per-element |Psi|^2 ratio for moving coordinate k of pos to xnew. */
int vmo_ratio(const vmo_system *s, const double *theta, const double *pos, int k, double xnew,
              double *ratios);

/* Philox4x32-10 (Salmon et al., SC'11): out = block(counter, key). */
void vmo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The engine's per-step random triple from Philox: stream tag 0, counter
 * {step_lo, step_hi, walker, 0}, key {seed_lo, seed_hi}.
 * out[0] = u_k in [0,1) (coordinate choice floor(u_k * D)),
 * out[1] = standard normal (IS) or uniform (BF),
 * out[2] = uniform in [0,1) for the accept test. */
void vmo_step_randoms(uint64_t seed, uint32_t walker, uint64_t step, int sampling, double out[3]);

/* Initial positions of one walker from Philox (stream tag 1):
 * RandomNormal N(0, sd) per coordinate (randomnormal.cpp:19 uses sd = 1/omega),
 * or RandomUniform U[0,1) (randomuniform.cpp:18). */
void vmo_initial_positions(uint64_t seed, uint32_t walker, int D, int normal, double sd,
                           double *pos);

/* Run `steps` Metropolis steps for W independent walkers.
 *  pos     W x D   in/out
 *  fcache  W x D   in/out: IS quantum-force cache (importancesampling.cpp:28-31)
 *  gpair   W x N x N in/out or NULL: per Pade pair, the gamma its cached f and h were
 *          last computed with (the reference refreshes a pair only when one of its
 *          particles makes an accepted move, padejastrow.cpp:65-68,192-209); NULL
 *          evaluates every pair with the current gamma.
 *  stream  W x steps x 3 replayed random triples, or NULL to use Philox(seed)
 *          with per-walker step counters `counter` (W entries, in/out).
 *  accepted W x steps (may be NULL)
 *  energies W x steps x 3 {T, Vext, Vint} per step (may be NULL)
 *  sums    W x (9 + 2*n_elem*p_max): per-walker accumulators over sampled steps
 *          {sum E, sum E^2, sum T, sum T^2, sum Vext, sum Vext^2, sum Vint,
 *           sum Vint^2, accepts, sum dlnPsi[n_elem*p_max], sum E*dlnPsi[...]}
 *  Steps i < burn_in are not sampled; the gradient window is
 *  bs*(iter % batches) < i < bs*(iter % batches + 1), bs = (steps-burn_in)/batches
 *  (sampler.cpp:82-83).
 * Returns 0, or <0 on a singular Slater block. */
int vmo_run(const vmo_system *s, const double *theta, int W, double *pos, double *fcache,
            double *gpair, int steps, int burn_in, int iter, int batches, const double *stream, uint64_t seed,
            uint64_t *counter, unsigned char *accepted, double *energies, double *sums);

/* Initial IS quantum-force cache F = 2 * sum_e grad_e at pos (importancesampling.cpp:28-31). */
int vmo_quantum_force(const vmo_system *s, const double *theta, const double *pos, double *f);

/* Blocking estimate of the variance of the mean (include/block/blocker.cpp:42-71).
 * n must be a power of two.  Returns the variance of the mean; *mean receives the mean. */
double vmo_blocking(const double *x, long n, double *mean);

#ifdef __cplusplus
}
#endif
#endif
