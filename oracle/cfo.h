/* CPU restatement of the reference's 3D SIMPLE hot path (ChuanFlow src/3d),
 * in plain C11, FP64, serial, compiled with -ffp-contract=off.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the parity tests check the
 * CUDA path against; the product never links or calls it.  Every function
 * follows the reference's operation order so that geometry, weights,
 * gradients, assembled matrices and right-hand sides come out bit-identical
 * to the reference's own CPU build (oracle/_ref), which is how this file is
 * pinned (tests/test_oracle_ref.py).
 *
 * Indices are int64 (the reference's `label`), reals are double (`scalar`).
 */
#ifndef CFO_H
#define CFO_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* boundary-condition kinds (src/3d/src/fields/volFields.cpp:117-147, :246-283) */
enum cfo_bc
{
    CFO_FIXED_VALUE = 0,
    CFO_ZERO_GRADIENT = 1,
    CFO_FIXED_GRADIENT = 2,
    CFO_SYMMETRY = 3,
    CFO_OUTLET = 4,
    CFO_WALL = 5,
    CFO_EMPTY = 6
};

/* gradient schemes (src/3d/src/discrete/gradScheme.cpp:246-277); any other
 * name behaves as CFO_GRAD_LINEAR */
enum cfo_grad
{
    CFO_GRAD_LINEAR = 0,
    CFO_GRAD_CORRECTED = 1,
    CFO_GRAD_LEAST_SQUARES = 2
};

enum cfo_div
{
    CFO_DIV_UPWIND = 0,
    CFO_DIV_LINEAR = 1,
    CFO_DIV_BLEND = 2,
    CFO_DIV_LINEAR_UPWIND = 3 /* this library's extension, no reference counterpart */
};

typedef struct cfo_mesh
{
    int64_t nP, nC, nF, nInt, nPatch;
    const double* pts;      /* nP*3 */
    const int64_t* fOff;    /* nF+1 */
    const int64_t* fV;      /* fOff[nF] */
    const int64_t* own;     /* nF */
    const int64_t* nbr;     /* nInt */
    const int64_t* pStart;  /* nPatch */
    const int64_t* pSize;   /* nPatch */
    /* geometry, filled by cfo_geometry (caller-owned storage) */
    double* V;       /* nC */
    double* C;       /* nC*3 */
    double* Cf;      /* nF*3 */
    double* Sf;      /* nF*3 */
    double* magSf;   /* nF */
    double* d;       /* nF*3 */
    double* invDist; /* nF */
} cfo_mesh;

/* boundary conditions of one SIMPLE case: per patch a type and a value for U
 * and p, plus optional per-face overrides (NULL = none) */
typedef struct cfo_bcs
{
    const int32_t* uType;   /* nPatch */
    const double* uValue;   /* nPatch*3 */
    const int32_t* pType;   /* nPatch */
    const double* pValue;   /* nPatch */
    const uint8_t* uFaceSet;  /* nF or NULL */
    const double* uFaceValue; /* nF*3 or NULL */
} cfo_bcs;

typedef struct cfo_controls
{
    int32_t maxIterations;
    double continuityTol, pcorrTol, momentumTol;
    double linearTol;
    int32_t linearMaxIter, nonOrthCorrectors;
    double relaxU, relaxP, pRelaxStart;
    double bodyForce[3];
    double nu;
    int32_t div, laplacianCorrected, grad;
    double blendCoeff;
    int32_t verbose;
    /* pressure reference cell (-1: none, the reference's behaviour); a pinned
     * cell follows OpenFOAM's fvMatrix::setReference: source += diag * value,
     * then diag += diag.  No counterpart in the reference. */
    int64_t pRefCell;
    double pRefValue;
    /* pressure preconditioner: 0 Jacobi (the reference), 1 multicolour DIC */
    int32_t pPrecond;
} cfo_controls;

typedef struct cfo_result
{
    int32_t iterations;
    int32_t converged;
    double finalContinuityError;
    double finalMomentumResidual;
    int32_t lastUIters, lastPIters;
    int32_t error;
    int64_t uItersTotal, pItersTotal; /* summed over components, passes, iterations */
} cfo_result;

typedef struct cfo_report
{
    int32_t iterations;
    int32_t converged;
    double initialResidual;
    double finalResidual;
} cfo_report;

/* blockMesh (src/3d/src/mesh/blockMesh.cpp:36-189) */
int cfo_block_counts(int64_t nx, int64_t ny, int64_t nz, int64_t out[4]);
int cfo_block_mesh(const double mn[3], const double mx[3], int64_t nx, int64_t ny, int64_t nz,
                   double* pts, int64_t* fOff, int64_t* fV, int64_t* own, int64_t* nbr,
                   int64_t* pStart, int64_t* pSize);

/* polyMesh::calcGeometry (src/3d/src/mesh/polyMesh.cpp:83-288) */
int cfo_geometry(cfo_mesh* m);
/* interpolate.cpp:15-48 */
void cfo_owner_weights(const cfo_mesh* m, double* ow);
void cfo_skew(const cfo_mesh* m, const double* ow, double* skew);
/* laplacianScheme.cpp:37-62 with a uniform cell gamma */
void cfo_harmonic_gamma(const cfo_mesh* m, double gamma, double* gf);

/* fvc::grad with explicit boundary face values bvals[f - nInt].  volQuirk
 * selects the volScalarField overload's internal face value for the plain
 * Gauss scheme (volFields.cpp:96-115); otherwise internal faces use the
 * bounded owner weight (interpolate.cpp:334-355). */
int cfo_grad(const cfo_mesh* m, const double* data, const double* bvals, int scheme, int volQuirk,
             double* out);

/* COO -> CSR (Matrix.cpp:56-117); returns nnz or -1; rowStart has n+1 */
int64_t cfo_csr_build(int64_t n, int64_t nTrip, const int64_t* rows, const int64_t* cols,
                      const double* vals, const double* diag, int64_t* rowStart, int64_t* outCols,
                      double* outVals);
void cfo_spmv(int64_t n, const int64_t* rowStart, const int64_t* cols, const double* vals,
              const double* x, double* y);
/* Matrix.cpp:153-222 and :224-319 */
int cfo_solve_cg(int64_t n, const int64_t* rowStart, const int64_t* cols, const double* vals,
                 const double* b, double* x, double tol, int32_t maxIter, cfo_report* rep);
int cfo_solve_bicgstab(int64_t n, const int64_t* rowStart, const int64_t* cols, const double* vals,
                       const double* b, double* x, double tol, int32_t maxIter, cfo_report* rep);

/* Multicolour DIC (no reference counterpart): greedy colouring, factor,
 * apply, and the PCG using it; see the definitions in cfo.c. */
int cfo_colour_cells(int64_t n, const int64_t* rs, const int64_t* cols, int32_t* colour);
int cfo_dic_factor(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const int32_t* colour,
                   int32_t nColours, double* rDinv);
void cfo_dic_apply(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const int32_t* colour,
                   int32_t nColours, const double* rDinv, const double* r, double* z);
int cfo_solve_dic_cg(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const double* b,
                     double* x, double tol, int32_t maxIter, cfo_report* rep);

/* solveIncompressibleSimple (simpleSolver.cpp:33-394), laminar, steady.
 * U (nC*3), p (nC), phi (nF) are updated in place. */
int cfo_simple(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, double* U, double* p,
               double* phi, cfo_result* res);

/* The assembly probes of oracle/ref_driver.cpp's `eqns` mode. */
int cfo_eqns(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, const double* U,
             const double* p, const double* phi, const double* xprobe, double* gradPn,
             double* uDiag /*3*nC*/, double* uH0 /*3*nC*/, double* uH1 /*3*nC*/, double* rAUf,
             double* divPhi, double* contErr, double* pDiag, double* pH0, double* pH1,
             double* gradPFull, double* phiCorrected);

/* updatePhiInternal + correctBoundaryFlux (pressureCorrection.cpp:10-25,
 * volFields.cpp:294-306) */
int cfo_flux_from_U(const cfo_mesh* m, const cfo_bcs* bc, const double* U, double* phi);

/* The pressure matrix (static laplacianFace part + reference cell) for a
 * given rAUf, as CSR; returns nnz. */
int64_t cfo_pressure_csr(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, const double* rAUf,
                         int64_t* rs, int64_t* cols, double* vals);

const char* cfo_last_error(void);

/* the library's device cell numbering (new -> old) for mode 0 identity,
 * 1 colour blocks, 2 reverse Cuthill-McKee, 3 colour blocks of RCM */
int cfo_cell_order(int64_t nC, int64_t nInt, const int64_t* own, const int64_t* nbr, int32_t mode,
                   int64_t* newToOld);

#ifdef __cplusplus
}
#endif
#endif
