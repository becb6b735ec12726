// Layout types shared by host and device code, and the checked CUDA call.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "cfg_internal.h"

namespace cfg
{

constexpr int TPB = 256;  // threads per block of every row/face kernel

// Coarse-correction scaling of the aggregation-AMG V-cycle (the piecewise
// constant prolongation undershoots, so its correction is scaled up): the
// pressure (Poisson-like) matrix and the momentum (upwind convection-
// diffusion) matrix each have their own.  On the 2M-cell channel the
// momentum BiCGStab needed 943.5, 928.1 and 1000.8 component-iterations per
// outer iteration with 2.0, 2.5 and 3.0.
constexpr float kAmgScalePressure = 2.0f;
constexpr float kAmgScaleMomentum = 2.5f;

#define CFG_CUDA(call)                                                                        \
    do                                                                                        \
    {                                                                                         \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            ::cfg::fail(CFG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

/// Three device arrays, one per vector component (structure of arrays).
struct V3P
{
    double* c[3];
};
struct CV3P
{
    const double* c[3];
};

/// Boundary linearisation face = c * cell + k for every boundary face and
/// component (volFields.cpp:117-147, :246-283), one table per field.
struct BcTab
{
    const double* c[3];
    const double* k[3];
};

/// Device mesh.  Face arrays are in the mesh's original face order; cell
/// arrays in device cell order (the identity unless renumbered).
struct DMesh
{
    int nC, nF, nI, nB;
    int nRowsPad;  // nC rounded up to a multiple of 32
    const int* own;   // nF
    const int* nbr;   // nI
    const double *sfx, *sfy, *sfz;  // face area vectors
    const double* ow;               // bounded owner weight (internal faces)
    const double* wq;               // volScalarField::faceValue weight (internal faces)
    const double *skx, *sky, *skz;  // skew vectors (internal faces)
    const double* oc;               // (Sf.d)/|d|^2
    const double* sfd;              // Sf.d
    const double* dd2;              // d.d
    const double *cvx, *cvy, *cvz;  // non-orthogonal vector Sf - dh (Sf.dh)
    const double* V;                // cell volumes
    const double* lscale;           // largest face area of each cell
    const double *cx, *cy, *cz;     // cell centres
    const double *fcx, *fcy, *fcz;  // face centres
    // cell -> faces, SELL-32 (slice-major, slot-major inside a slice): each
    // cell's faces in ascending original face order; code = face<<1 | side
    // (side 1: the cell is the face's neighbour), -1 pads; other = the cell
    // across an internal face or the boundary index of a boundary face
    const int* cfStart;  // nSlices+1, in entries
    const int* cfCode;
    const int* cfOther;
    // matrix rows, SELL-32: entries in the reference CSR's column order with
    // the diagonal in place; code = face<<1|side, -2 diagonal, -1 pad
    const int* mStart;
    const int* mCol;
    const int* mCode;
};

/// Device state of one Jacobi-PCG or 3-component BiCGStab solve.
struct SolveState
{
    double tol;
    int maxIter;
    int nComp;
    // per component
    double bnorm[3], init[3], fin[3];
    double rho[3], alpha[3], omega[3], beta[3];
    double rz[3], pAp[3];
    int it[3], done[3], conv[3], special[3];
    int allDone;
    int normType;  // 0: |r|inf / |b|inf (the reference's test); 1: |r|2 / |b|2
    unsigned int ticket[8];
};

/// Multicolour DIC layout (see dic.cuh).
template <class T>
struct DDicT
{
    int nColours;
    const int* rows;      // cells grouped by colour, ascending within a colour
    const int* lStart;    // lower SELL: slice offsets (all colours, concatenated)
    const int* lCol;
    const int* lSrc;      // index of the entry in the main matrix SELL
    const int* uStart;    // upper SELL
    const int* uCol;
    const int* uSrc;
    T* lVal;
    T* uVal;
    T* rD;
    T* rDinv;
};
using DDic = DDicT<double>;

/// one colour: cnt rows starting at rows[off], slices starting at slice0
struct DicPhase
{
    int off, cnt, slice0, partialOff;
};

}  // namespace cfg
