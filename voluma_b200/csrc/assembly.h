// Device-resident mesh geometry and the finite-volume assembly kernels of the pressure
// equation: fvm::laplacian (with explicit non-orthogonal correction), fvc::grad (Gauss linear,
// weighted least squares), fvc::div, the FvMatrix boundary fold / setReference / flux, and the
// non-orthogonal-corrector loop of the pressure equation around the GAMG-PCG solve.
#pragma once

#include <cstdint>
#include <vector>

#include "common.h"
#include "solver.h"

namespace vlm {

// Scalar boundary conditions of one field: per patch 0 = zeroGradient (also a scalar symmetry plane),
// 1 = fixedValue, 4 = mixed with refGrad 0 (value fraction per face in `frac`, reference value in
// `value`; freestreamPressure), 5 = fixedGradient (the gradient in `value`); values per boundary
// face, index f - nInternal.
struct ScalarBC {
    const int32_t* type = nullptr;  // host, nPatches
    const double* value = nullptr;  // device, nBoundary (may be null: 0)
    const double* frac = nullptr;   // device, nBoundary: value fractions of type-4 faces
    const int32_t* lsFix = nullptr; // device, nPatches: least-squares value constraint (Fvc.h:267-287,
                                    // bc.fixesValue()); null: the fixedValue patches (and Robin with a != 0)
    const double* robin = nullptr;  // device, nPatches x {a, b}: Robin (type 8) a phi + b dphi/dn = value
};

class DeviceGeom {
public:
    // Host arrays of cfd::Mesh (see vlm_mesh_desc); copied to the device.
    DeviceGeom(int nCells, int nInternal, int nFaces, const int32_t* own, const int32_t* nei, const double* magSf,
               const double* ndc, const double* V, const double* Sf, const double* d, const double* w,
               const double* corrVecs, int twoD, int emptyDir, int nPatches, const int32_t* patchStart,
               const int32_t* patchSize, const double* C, const double* Cf, const double* skewVecs,
               cudaStream_t stream);

    int nCells() const { return nC_; }
    int nInternal() const { return nI_; }
    int nFaces() const { return nF_; }
    int nBoundary() const { return nF_ - nI_; }
    bool nonOrthogonal() const { return nonOrth_; }
    bool skewed() const { return skewed_; }
    bool hasSkewVectors() const { return skew_.size() > 0; }  // Mesh::skewed(); skew() is then the SoA x_f - x'_f

    // fvm::laplacian(gamma, psi) for a scalar field (Fvm.h:141-182).  All pointers device.
    // gradScheme: 0 Gauss linear, 1 least squares.  ffc may be null when not needed.
    void laplacian(const double* gamma, const double* psi, const double* psiB, const ScalarBC& bc, bool nonOrthCorr,
                   int gradScheme, double* diag, double* upper, double* source, double* ic, double* bs, double* ffc,
                   bool* hasFfc, cudaStream_t s);

    // fvc::grad of a scalar (Fvc.h:209-291), scheme 0 Gauss linear, 1 leastSquares, 2 GaussSkew (needs
    // the skew vectors): out 3*nCells (x,y,z per cell).  psiB: boundary values.
    void grad(const double* psi, const double* psiB, const ScalarBC& bc, int scheme, double* out, cudaStream_t s);

    // zeroGradient / fixedValue boundary values of a scalar field (correctBoundaryConditions)
    void correctBoundary(const double* psi, const ScalarBC& bc, double* psiB, cudaStream_t s);

    // FvMatrix::solve's fold (FvMatrix.h:154-163): d = diag + Σ ic, b = source + Σ bs
    void fold(const double* diag, const double* source, const double* ic, const double* bs, double* d, double* b,
              cudaStream_t s);

    // FvMatrix::flux (FvMatrix.h:210-222), symmetric matrix: F = upper psi_N - upper psi_P (+ffc)
    void flux(const double* upper, const double* psi, const double* ic, const double* bs, const double* ffc,
              double* F, cudaStream_t s);

    // source += su * V  (FvMatrix::operator-=(su), FvMatrix.h:93-97)
    void addVolumeSource(double* source, const double* su, cudaStream_t s);

    // fvc::div(F) (Fvc.h:294-304): per unit volume
    void div(const double* F, double* out, cudaStream_t s);

    // setReference (FvMatrix.h:134-141) on one cell / on n cells (device list of global cells)
    void setReference(int cell, double value, double* diag, double* source, cudaStream_t s);
    void setReferences(const int32_t* cells, int n, double value, double* diag, double* source, cudaStream_t s);

    // gather list of one cell's faces: [cfOff[c], cfOff[c+1]) entries f | (cell is neighbour) << 31
    const int32_t* cellFaceOff() const { return cfOff_.get(); }
    const int32_t* cellFaces() const { return cfList_.get(); }

    // raw device arrays (vectors SoA: [x(n) y(n) z(n)]) for the momentum kernels
    const int32_t* own() const { return own_.get(); }
    const int32_t* nei() const { return nei_.get(); }
    const int32_t* bPatch() const { return bPatch_.get(); }
    const double* magSf() const { return magSf_.get(); }
    const double* ndc() const { return ndc_.get(); }
    const double* V() const { return V_.get(); }
    const double* w() const { return w_.get(); }
    const double* Sf() const { return Sf_.get(); }
    const double* d() const { return d_.get(); }
    const double* corr() const { return corr_.get(); }
    const double* C() const { return C_.size() ? C_.get() : nullptr; }
    const double* Cf() const { return Cf_.size() ? Cf_.get() : nullptr; }
    const double* skew() const { return skewed_ ? skew_.get() : nullptr; }  // null on unskewed meshes
    int twoD() const { return twoD_; }
    int64_t launches() const { return launches_; }  // kernels launched by the methods above
    int emptyDir() const { return emptyDir_; }
    int nPatches() const { return int(patchStart_.size()); }
    const std::vector<int32_t>& patchStart() const { return patchStart_; }
    const std::vector<int32_t>& patchSize() const { return patchSize_; }

private:
    int nC_, nI_, nF_, twoD_, emptyDir_;
    bool nonOrth_ = false, skewed_ = false;
    std::vector<int32_t> patchStart_, patchSize_, bPatchHost_;
    DBuf<int32_t> own_, nei_, cfOff_, cfList_, bPatch_, bcType_;
    std::vector<int32_t> bcTypeHost_;  // the patch types last copied to bcType_
    DBuf<double> magSf_, ndc_, V_, w_, Sf_, d_, corr_;  // vectors as SoA: [x(nF) y(nF) z(nF)]
    DBuf<double> C_, Cf_, skew_;                        // SoA; empty when not registered (skew_: not skewed)
    int64_t launches_ = 0;
    DBuf<double> scratchG_, scratchGS_, scratchGls_;
    void uploadBCType(const ScalarBC& bc, cudaStream_t s);
};

}  // namespace vlm
