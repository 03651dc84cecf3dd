// intg.cuh -- device-side system description, work lists and kernel
// launchers of the B200 integral setup.
#pragma once

#include <vector>

#include "common.cuh"

namespace imago {

// Everything the kernels read about the system, as device pointers.
struct DevSys {
  int nt, ns, npt, nps, nk, ncell;
  int vale_dim, core_dim;
  double T;            // logBasisFnThresh = -ln(basisFnConvg)
  double rv[9];        // realVectors [abc*3 + xyz]
  double inv[9];       // invRealVectors [abc*3 + xyz]
  // 1.5 x the smallest singular value of realVectors: every lattice point
  // outside the 3x3x3 block around a rounded point is at least this far
  double far_lattice;
  // every k-point is Gamma: all phases are exactly 1, every matrix is real,
  // and the orthogonalisation runs on the real parts only
  int real_k;
  // the phase sum multiplies by -i (applyPhaseFactors runCode 1,
  // intgSaving.F90:178-186): the momentum matrix -i<a|d/dx|b> is Hermitian
  int minus_i;
  // atom types
  const int *type_nalpha, *type_alpha_off, *type_nstates, *type_nvale,
      *type_state_off, *type_basis_off, *type_screen;
  const double *alpha;
  const int *alpha_cls;   // 0..3
  const int *state_lm;    // 0-based lm per state
  const double *basis;    // [basis_off + a * nstates + m]
  // atom sites
  const double *site_pos;
  const int *site_type, *site_cum_vale, *site_cum_core;
  // potential types and sites
  const double *ptype_z, *ptype_nucalpha, *palpha;
  const int *ptype_alpha_off, *ptype_nalpha, *ptype_first_site, *ptype_mult,
      *ptype_screen;
  const double *psite_pos;
  const int *psite_ptype;
  // lattice cells sorted by |R|^2, k-points, phase table
  const double *cell;     // [n*3]
  const double *csize;    // [n]
  const double *kxyz;     // [nk*3]
  const double2 *phase;   // [cell * nk + k]  exp(i k.R)
  // device status word: a kernel whose bounded wait ran out records
  // IMAGO_ERR_TIMEOUT here (first failure wins); read after each call
  int *flag;
};

// Atom pair (i <= j) that passes the nearest-image screen.
struct DPair {
  int i, j, ti, tj;
  int ni, nj;             // total states of the two atoms
  int ubeg, uend;         // units [ubeg, uend)
  double L0[3];           // nearest lattice vector to pos_i - pos_j
  long long moff;         // first element of the pair's unit blocks
};

// (pair, lattice image) within the pair cutoff.
struct DUnit {
  int pair, cell;
  int spbeg, spend;       // shell pairs [spbeg, spend), staircase order
  double r2;              // |A - B'|^2
};

// Screened primitive pair of one unit.
struct DSp {
  int unit;
  short a, b;             // alpha indices (0-based)
  short la, lb;           // classes
  long long boff;         // offset of its sh block in a term's block buffer
};

struct DevWork {
  int npairs, nunits, nsp;
  const DPair *pairs;
  const DUnit *units;
  const DSp *sps;
  const int *sp_by_cls;   // shell pairs sorted by class (la*4+lb), then unit
  long long blk_total;    // doubles of sh blocks per term
  long long m_total;      // doubles of unit blocks per term
  int nbtile;             // phase-sum column tiles of kBlochCols: (pair, tile)
  const int2 *btile;
  int bw;                 // column width of the tensor-core phase sum
  int nbtile_w;           // its tiles: (pair, tile of bw columns)
  const int2 *btile_w;
  // [unit * nps + site]: the potential site's nearest image to the midpoint
  // of the unit's A-B segment (null: every site is searched in full)
  const struct SiteImage *simg;
  // [unit * ncl + c]: the smallest d1 of sites kSiteCluster*c .. +7 (null
  // with simg)
  const float *cl_d1;
  int ncl;
  // [unit * nps + first site of type + r]: the r-th site of the type in
  // ascending d1 for that unit, as an offset within the type (null with
  // simg)
  const int *site_rank;
};

// Consecutive potential sites screened together before their own tests.
constexpr int kSiteCluster = 8;

// Nearest image of a potential site C to the midpoint M of a unit's A-B
// segment: M - C - (n0 a + n1 b + n2 c) is shortest for lattice coordinates
// n; d1 and d2 are lower bounds of the distance from M - C to that lattice
// point and to every other one.  16 bytes, so that the table of a large
// cell stays compact.
struct __align__(16) SiteImage {
  short n[3];
  short pad;
  float d1, d2;
};

// Columns (block elements) per CTA of the register phase sum, and the
// column widths the tensor-core phase sum is tuned over (32, 48, 64).
constexpr int kBlochCols = 64;
constexpr int kNumBlochWidths = 3;
__host__ __device__ constexpr int bloch_width(int i) { return 32 + 16 * i; }
// Up to this many k-points the phase sum keeps its sums in registers.
constexpr int kBlochSmallNk = 8;

// Term of a three-centre build: NP is one term over all sites; EP term j of
// potential type t has alpha index j.
struct Term3c {
  int nuclear;            // 1: NP
  int ptype, j;           // EP only
};

// Two-centre primitive operators of launch_prim2c.
enum { kPrim2cOverlap = 0, kPrim2cKinetic = 1, kPrim2cMassVel = 2 };

// The library's stream-ordered device memory pool of the current device
// (freed memory stays in it until imago_trim_memory); null if none.
cudaMemPool_t device_scratch_pool();

// Launchers (kernels.cu).  All take the stream to run on.
int launch_prim2c(const DevSys &s, const DevWork &w, const int *cls_beg,
                  int op, double *blk, cudaStream_t st);
// The PSCF Hamiltonian's potential terms for one spin, summed in registers
// per shell pair: H = sum_t coef[t] EP_t (sh blocks, written, not added).
// lanes (1 or 4) threads share a shell pair's terms (s, p, d classes).
int launch_prim3c_ham(const DevSys &s, const DevWork &w, const int *cls_beg,
                      const Term3c *terms_dev, int nterm, const double *coef,
                      int lanes, double *H, cudaStream_t st);
// The three wave vectors of a K-overlap build, q[3 * axis + xyz].
struct KovWaves {
  double q[9];
};
// K-overlap primitive blocks: real and imaginary parts of axis a as terms
// 2a and 2a + 1 (blk + t * blk_total).
int launch_prim_kov(const DevSys &s, const DevWork &w, const int *cls_beg,
                    const KovWaves &dk, double *blk, cudaStream_t st);
// The K-overlap's complex phase sum (M: 6 real terms) with the full saving
// of the reference (block (j, i) the dagger of block (i, j), a diagonal
// block replaced by its dagger): vv/cv/cc hold 3 complex terms.
int launch_bloch_kov(const DevSys &s, const DevWork &w, const double *M, double2 *vv,
                     double2 *cv, double2 *cc, cudaStream_t st);
// The K-overlap's orthogonalisation on the full matrix, no Hermitian form:
// W = VV - S^H X_cv - X_cv^H S + S^H X_cc S, 3 terms, written as real and
// imaginary [term][k][col][row] planes.
int launch_ortho_full(const DevSys &s, const double2 *vv, const double2 *cv,
                      const double2 *cc, const double2 *s_cv, double2 *y, double *re,
                      double *im, cudaStream_t st);
// Momentum (dipole = false) or dipole blocks about `center`: three
// components per shell pair, component c at blk + c * blk_total.
int launch_prim2c_vec(const DevSys &s, const DevWork &w, const int *cls_beg,
                      bool dipole, const double center[3], double *blk,
                      cudaStream_t st);
// The classes of one three-centre build in work-queue order: class code
// la * 4 + lb, first entry of its shell-pair list, count, and the first
// queue item of each class (off[ncls] is the total).
// Consecutive EP terms of one potential type evaluated by one thread, so
// that they share the site and image walk: group g is terms first[g] ..
// first[g] + count[g] - 1 of a launch's term list.
constexpr int kMaxTermGroups = 64;
struct TermGroups {
  int n;
  unsigned short first[kMaxTermGroups];
  unsigned char count[kMaxTermGroups];
};
// Pairs of consecutive terms of one type (a single term where a type's
// count is odd); n = 0 when there would be more than kMaxTermGroups.
TermGroups term_pairs(const Term3c *terms_host, int nterm);

struct Prim3cQueue {
  int ncls;
  int cls[16], beg[16], n[16];
  long long off[17];
};

// All classes of a three-centre build in one persistent launch of `ctas`
// CTAs fed by a device counter (8 bytes at `counter`, zeroed here on the
// stream before the launch).
int launch_prim3c_queue(const DevSys &s, const DevWork &w, const int *cls_beg,
                        const Term3c *terms_dev, int nterm, bool nuclear, double *blk,
                        unsigned long long *counter, int ctas, cudaStream_t st);
// CTAs of k_prim3c_queue resident per SM.
int prim3c_queue_ctas_per_sm();
// Screened (shell pair, site, image) triples of the s/p/d classes into
// count16[la * 4 + lb] (added), by the count-only form of k_prim3c.
int launch_prim3c_count(const DevSys &s, const DevWork &w, const int *cls_beg,
                        const Term3c *terms_dev, int nterm, bool nuclear,
                        unsigned long long *count16, cudaStream_t st);

// terms_host (the same list on the host): EP classes up to d-p run two
// terms of a type per thread (k_prim3c_pair); null: one term per thread.
int launch_prim3c(const DevSys &s, const DevWork &w, const int *cls_beg,
                  const Term3c *terms_dev, int nterm, bool nuclear,
                  double *blk, cudaStream_t st, const Term3c *terms_host = nullptr);
// terms_per_cta: 4 or 8 EP terms per CTA (builds of up to 4 terms use 4)
int launch_contract(const DevSys &s, const DevWork &w, int nterm,
                    const double *blk, double *M, cudaStream_t st, int terms_per_cta = 4);
int launch_bloch(const DevSys &s, const DevWork &w, int nterm, const double *M,
                 double2 *vv, double2 *cv, double2 *cc, cudaStream_t st);
// pipe: the persistent TMA-fed kernel where it applies (several terms,
// S and two X_cv buffers in shared memory), the per-(k, term) CTAs else.
int launch_ortho(const DevSys &s, int nterm, const double2 *vv,
                 const double2 *cv, const double2 *cc, const double2 *s_cv,
                 double2 *y, double *packed, cudaStream_t st, bool pipe = false);
bool ortho_pipe_fits(int C, int V);
// One CTA waiting (bounded, limit_ms) on a barrier nothing completes; it
// records IMAGO_ERR_TIMEOUT in *flag.
int launch_wait_check(int *flag, double limit_ms, cudaStream_t st);
// The same for a matrix whose core-core block is not Hermitian (dipole):
// the reference's zher2k-then-makeValeVale sequence as it stands.
int launch_ortho_general(const DevSys &s, int nterm, const double2 *vv,
                         const double2 *cv, const double2 *cc,
                         const double2 *s_cv, double2 *y, double *packed,
                         cudaStream_t st);
// H[q] += sum_t w(t, q) blk[t] over the sh blocks of one term each
// (n doubles), for the PSCF Hamiltonian.
int launch_block_axpy(const double *blk, int nterm, long long n, const double *w,
                      int wstride, int spin, double *H, cudaStream_t st);
int launch_split_cv(const DevSys &s, const double2 *cv, double *re, double *im,
                    cudaStream_t st);
int launch_phase(const DevSys &s, double2 *phase, cudaStream_t st);
int launch_site_images(const DevSys &s, const DevWork &w, SiteImage *simg,
                       float *cl_d1, cudaStream_t st);
int launch_prim_eval(int kind, int n, const double *params, const int *cls,
                     double *sh, cudaStream_t st);

// makeValenceRho's traces of packed matrices against packed densities
// (k_secular.cu); `part` holds packed_traces_work(...) doubles.
size_t packed_traces_work(int vale_dim, int nk, int nmat, int nrho);
int launch_packed_traces(int vale_dim, int nk, int nmat, const double *mats, int nrho,
                         const double *rho, double *part, double *traces, cudaStream_t st);

}  // namespace imago
