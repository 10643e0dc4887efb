// pppm_compat.hpp — C++ classes with the reference's interface for the PPPM
// path, implemented over the C ABI in pppm.h (header only; link
// libpppm_b200.so).
//
//   BiotSavartSolver              hybridFastSummation/BiotSavartSolver.h:16-38
//   ParticleManager               particle_hash/SpaceHashClass.h:10-84
//   MultiGridSolver3DPeriod_double multigrid/MultiGrid.h:188-209
//   PotentialFieldSolver          hybridFastSummation/PotentialFieldSolver.h:10-91
//
// The reference passes gf::gf_GpuArray<T> objects (multigrid/gfGpuArray.h:
// 26-89); DeviceArray<T> below keeps the members its call sites use,
// getDevicePtr(), getSize() and typeSize(), over device memory owned by the
// caller or by the solver.  Element types are the CUDA vector types the
// reference uses (float4 positions, double4 origin, double3 gradients), so
// its call expressions — getU(0)->getDevicePtr(), getSortPos()->getDevicePtr(),
// getOrigin().x — compile unchanged.  Methods return bool like the reference,
// but false on failure (the reference always returns true and exits on CUDA
// errors); lastError() gives the reason.
#pragma once

#include <cuda_runtime.h>  // float4, double4, double3, float3, uint3

#include <cstdint>
#include <cstring>
#include <string>

#include "pppm.h"

namespace pppm_compat {

typedef unsigned int uint;

// Earlier spellings of the element types, kept as aliases.
typedef float4 float4_;
typedef double4 double4_;
typedef double3 double3_;

template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(T *dev, size_t n) : ptr_(dev), n_(n) {}
    T *getDevicePtr() const { return ptr_; }
    size_t getSize() const { return n_; }
    size_t typeSize() const { return sizeof(T); }

private:
    T *ptr_ = nullptr;
    size_t n_ = 0;
};

typedef DeviceArray<float4> GpuArrayf4;
typedef DeviceArray<double> GpuArrayd;
typedef DeviceArray<double3> GpuArrayd3;

inline std::string lastError() { return pppm_last_error(); }

class BiotSavartSolver {
public:
    BiotSavartSolver() = default;
    ~BiotSavartSolver() { shutdown(); }
    BiotSavartSolver(const BiotSavartSolver &) = delete;
    BiotSavartSolver &operator=(const BiotSavartSolver &) = delete;

    // HFS/BiotSavartSolverImp.cpp:44-229.  Cubic grids only; isVIC (mesh-only
    // velocities) is not part of this path and is rejected.
    bool initializeSolver(uint gdx, uint gdy, uint gdz, bool isVIC, int K, uint M, uint N,
                          void *stream = nullptr) {
        if (gdx != gdy || gdy != gdz || isVIC) return false;
        if (scene_ && gdx == n_ && K == K_) {
            M_ = M;
            N_ = N;
            return true;
        }
        shutdown();
        pppm_params p;
        pppm_params_default(&p);
        p.n = gdx;
        p.K = K;
        if (pppm_scene_create(&p, N ? N : 1, M ? M : 1, stream, &scene_) != PPPM_OK) return false;
        n_ = gdx;
        K_ = K;
        M_ = M;
        N_ = N;
        return true;
    }

    // HFS/BiotSavartSolverImp.cpp:318-360
    bool setVortParameter(uint n, GpuArrayf4 *pos, GpuArrayd *omega[]) {
        N_ = n;
        sorted_valid_ = false;
        for (int c = 0; c < 3; c++) vort_arr_[c] = GpuArrayd(omega[c]->getDevicePtr(), n);
        return pppm_set_vortices(scene_, n, reinterpret_cast<const float *>(pos->getDevicePtr()),
                                 vort_arr_[0].getDevicePtr(), vort_arr_[1].getDevicePtr(),
                                 vort_arr_[2].getDevicePtr()) == PPPM_OK;
    }

    // HFS/BiotSavartSolverImp.cpp:266-316
    bool setEvalParameter(uint m, GpuArrayf4 *pos) {
        M_ = m;
        eval_ = reinterpret_cast<const float *>(pos->getDevicePtr());
        return ensure_u(m);
    }

    // HFS/BiotSavartSolverImp.cpp:756-816
    void computeFarFieldBuffer() { ok_ = pppm_build_far_field(scene_) == PPPM_OK; }

    // HFS/BiotSavartSolverImp.cpp:410-516
    bool evaluateVelocity(GpuArrayf4 *another_end, uint is_segment) {
        const float *eb = another_end ? reinterpret_cast<const float *>(another_end->getDevicePtr()) : nullptr;
        return pppm_eval(scene_, M_, eval_, eb, (int)is_segment, U_[0], U_[1], U_[2]) == PPPM_OK;
    }

    // HFS/BiotSavartSolver.h:24-27: the solver's own arrays, valid until the
    // next call that resizes them or shutdown().
    GpuArrayd *getU(int i) { return &u_arr_[i]; }
    GpuArrayd *getVort(int i) { return &vort_arr_[i]; }

    // HFS/BiotSavartSolverImp.cpp:733-753: hash + reorder; the sorted copies are
    // produced on request by getSortPos / getSortVort.
    void sortVort() {
        ok_ = pppm_build_far_field(scene_) == PPPM_OK;
        sorted_valid_ = false;
    }
    GpuArrayf4 *getSortPos() { return refresh_sorted() ? &spos_arr_ : nullptr; }
    GpuArrayd *getSortVort(int i) { return refresh_sorted() ? &salpha_arr_[i] : nullptr; }

    // HFS/BiotSavartSolver.h:28-29 (n^3 entries; empty cells hold 0xFFFFFFFF)
    uint *getVortStartTable() {
        const uint32_t *s = nullptr, *e = nullptr;
        pppm_get_cell_tables(scene_, &s, &e);
        return const_cast<uint *>(s);
    }
    uint *getVortEndTable() {
        const uint32_t *s = nullptr, *e = nullptr;
        pppm_get_cell_tables(scene_, &s, &e);
        return const_cast<uint *>(e);
    }
    double getCellh() {
        double o[3], L = 0, h = 0;
        pppm_get_domain(scene_, o, &L, &h);
        return h;
    }
    double4 getOrigin() {
        double o[3] = {0, 0, 0}, L = 0, h = 0;
        pppm_get_domain(scene_, o, &L, &h);
        return make_double4(o[0], o[1], o[2], 0.0);
    }

    // HFS/BiotSavartSolverImp.cpp:230-264
    bool shutdown() {
        if (scene_) pppm_scene_destroy(scene_);
        scene_ = nullptr;
        free_buffers();
        return true;
    }

    bool lastOk() const { return ok_; }
    pppm_scene *scene() { return scene_; }

private:
    // Output arrays are owned by the solver, as m_particle_U is in the
    // reference; they are allocated with the CUDA runtime the application
    // links (cudaMalloc), outside the library.
    bool ensure_u(uint m);
    bool refresh_sorted();
    void free_buffers();

    pppm_scene *scene_ = nullptr;
    uint n_ = 0, M_ = 0, N_ = 0, capU_ = 0, capS_ = 0;
    int K_ = 1;
    const float *eval_ = nullptr;
    double *U_[3] = {nullptr, nullptr, nullptr};
    float4 *spos_ = nullptr;
    double *salpha_[3] = {nullptr, nullptr, nullptr};
    GpuArrayd u_arr_[3], vort_arr_[3], salpha_arr_[3];
    GpuArrayf4 spos_arr_;
    bool sorted_valid_ = false;
    bool ok_ = true;
};

class MultiGridSolver3DPeriod_double {
public:
    ~MultiGridSolver3DPeriod_double() { m_FinalMemoryEachLevel(); }
    // MG/MultiGrid.h:129-139
    void m_InitialSystem(int gridx, int gridy, int gridz, void *stream = nullptr) {
        m_FinalMemoryEachLevel();
        if (gridx == gridy && gridy == gridz) pppm_mg_create((uint32_t)gridx, stream, &mg_);
    }
    void m_FinalMemoryEachLevel() {
        if (mg_) pppm_mg_destroy(mg_);
        mg_ = nullptr;
    }
    // MG/MultiGrid.cpp:202-250 (tol ignored in the reference schedule)
    void m_FullMultiGrid(GpuArrayd *x, GpuArrayd *b, double tol, double &residual) {
        double rr = -1.0;
        pppm_mg_full_multigrid(mg_, x->getDevicePtr(), b->getDevicePtr(), PPPM_MG_REFERENCE, tol, 1, &rr);
        residual = rr;
    }
    // MG/MultiGrid.cpp:128-201: one V(4,4) cycle from `level` down, on that
    // level's arrays (level 0 = the full grid).  As in the reference, tol is
    // not used and residual is left as it is.
    void m_Vcycle(GpuArrayd *x, GpuArrayd *b, double /*tol*/, double & /*residual*/, int level) {
        pppm_mg_vcycle(mg_, x->getDevicePtr(), b->getDevicePtr(), level);
    }

private:
    pppm_mg *mg_ = nullptr;
};

class ParticleManager {
public:
    ParticleManager() = default;
    // PH/SpaceHashClassImp.cpp:6-14: a 64^3 grid of cell size 1/64 at the
    // origin; device tables come with initSpatialHash.
    explicit ParticleManager(uint numParticles) : N_(numParticles) {}
    ~ParticleManager() { endSpatialHash(); }
    ParticleManager(const ParticleManager &) = delete;
    ParticleManager &operator=(const ParticleManager &) = delete;
    // PH/SpaceHashClassImp.cpp:47-69
    void initSpatialHash(uint numParticles, uint dimx, uint dimy, uint dimz, void *stream = nullptr) {
        endSpatialHash();
        if (dimx == dimy && dimy == dimz) pppm_hasher_create(numParticles, dimx, stream, &h_);
        n_ = dimx;
        h_cell_ = 1.0f / (float)dimx;
    }
    void endSpatialHash() {
        if (h_) pppm_hasher_destroy(h_);
        h_ = nullptr;
    }
    // PH/SpaceHashClass.h:46-54
    void setSpatialHashGrid(uint size0, float h, float3 bbmin, uint numParticles) {
        n_ = size0;
        h_cell_ = h;
        origin_[0] = bbmin.x;
        origin_[1] = bbmin.y;
        origin_[2] = bbmin.z;
        N_ = numParticles;
    }
    void setHashParam() {}  // parameters travel with each call
    void doSpatialHash(float4 *pos, uint numParticles) {
        pppm_hasher_run(h_, numParticles, reinterpret_cast<const float *>(pos), h_cell_, origin_);
    }
    void reorderData(uint numParticles, void *data, void *dataReorder, uint stride, uint precision) {
        pppm_hasher_reorder(h_, numParticles, data, dataReorder, stride, precision);
    }
    void deorderData(uint numParticles, void *data, void *dataReorder, uint stride, uint precision) {
        pppm_hasher_deorder(h_, numParticles, data, dataReorder, stride, precision);
    }
    // PH/SpaceHashClass.h:24-38, 67-69
    uint *getHashTable() { return const_cast<uint *>(table(0)); }
    uint *getStartTable() { return const_cast<uint *>(table(2)); }
    uint *getEndTable() { return const_cast<uint *>(table(3)); }
    int getNumParticles() const { return (int)N_; }
    uint3 getGridSize() const { return make_uint3(n_, n_, n_); }
    float3 getWorldOrigin() const { return make_float3(origin_[0], origin_[1], origin_[2]); }
    float3 getCellSize() const { return make_float3(h_cell_, h_cell_, h_cell_); }
    uint getNumCells() const { return n_ * n_ * n_; }

private:
    const uint32_t *table(int which) {
        const uint32_t *t[4] = {nullptr, nullptr, nullptr, nullptr};
        pppm_hasher_tables(h_, &t[0], &t[1], &t[2], &t[3]);
        return t[which];
    }
    pppm_hasher *h_ = nullptr;
    uint n_ = 64, N_ = 0;
    float h_cell_ = 1.0f / 64.0f;
    float origin_[3] = {0.f, 0.f, 0.f};
};

// HFS/PotentialFieldSolver.h:10-91.  Output arrays are owned by the solver, as
// m_particle_gradPhi / m_particle_dphidn are in the reference.
class PotentialFieldSolver {
public:
    PotentialFieldSolver() = default;
    ~PotentialFieldSolver() { shutdown(); }
    PotentialFieldSolver(const PotentialFieldSolver &) = delete;
    PotentialFieldSolver &operator=(const PotentialFieldSolver &) = delete;

    // :45-255 (cubic grids only)
    bool initializeSolver(uint gdx, uint gdy, uint gdz, uint K, uint M, uint N, void *stream = nullptr) {
        if (gdx != gdy || gdy != gdz) return false;
        shutdown();
        if (pppm_potential_create(gdx, (int)K, N ? N : 1, M ? M : 1, stream, &p_) != PPPM_OK) return false;
        n_ = gdx;
        return true;
    }
    // :344-392
    bool setMassParameter(uint n, GpuArrayf4 *pos, GpuArrayd *mass) {
        mass_ = mass->getDevicePtr();
        return pppm_potential_set_masses(p_, n, reinterpret_cast<const float *>(pos->getDevicePtr()),
                                         mass->getDevicePtr()) == PPPM_OK;
    }
    // :302-343
    bool setEvalParameter(uint m, GpuArrayf4 *pos) {
        M_ = m;
        eval_ = reinterpret_cast<const float *>(pos->getDevicePtr());
        return ensure_out(m);
    }
    bool setEvalNormals(uint, GpuArrayd3 *normals) { normals_ = normals->getDevicePtr(); return true; }
    bool setEvalAreas(uint, GpuArrayd *areas) { areas_ = areas->getDevicePtr(); return true; }
    // :695-707
    void computeFarFieldBuffer() { ok_ = pppm_potential_build(p_, 0) == PPPM_OK; }
    // :726-737
    void computeFarFieldPotentialBuffer() { ok_ = pppm_potential_build(p_, 1) == PPPM_OK; }
    // :441-526 (large_eval only changes the reference's evaluation order)
    bool evaluateGradient(bool /*large_eval*/) {
        return pppm_potential_eval_gradient3(p_, M_, eval_, reinterpret_cast<double *>(grad_)) == PPPM_OK;
    }
    // :708-739
    void evaluateScalarPotential() { ok_ = pppm_potential_eval_scalar(p_, M_, eval_, dphidn_) == PPPM_OK; }
    // :621-626; normals and gradients as double3 records
    bool computeDphiDn();
    GpuArrayd3 *getGradPhi() { grad_arr_ = GpuArrayd3(grad_, M_); return &grad_arr_; }
    GpuArrayd *getDpDn() { dp_arr_ = GpuArrayd(dphidn_, M_); return &dp_arr_; }
    GpuArrayd *getScalarPhi() { return getDpDn(); }
    double getCellh() {
        double ol[4] = {0, 0, 0, 0};
        pppm_potential_grids(p_, ol, nullptr, nullptr, nullptr, nullptr, nullptr);
        return (double)(float)(ol[3] / (double)n_);
    }
    double4 getOrigin() {
        double ol[4] = {0, 0, 0, 0};
        pppm_potential_grids(p_, ol, nullptr, nullptr, nullptr, nullptr, nullptr);
        return make_double4(ol[0], ol[1], ol[2], 0.0);
    }
    bool shutdown();
    bool lastOk() const { return ok_; }

private:
    bool ensure_out(uint m);
    pppm_potential *p_ = nullptr;
    uint n_ = 0, M_ = 0, cap_ = 0;
    const float *eval_ = nullptr;
    const double *mass_ = nullptr, *areas_ = nullptr;
    const double3 *normals_ = nullptr;
    double3 *grad_ = nullptr;
    double *dphidn_ = nullptr, *split_ = nullptr;  // split_: [6][cap] SoA scratch for computeDphiDn
    GpuArrayd3 grad_arr_;
    GpuArrayd dp_arr_;
    bool ok_ = true;
};

}  // namespace pppm_compat

// Out-of-line members that allocate: kept here so the header stays self
// contained; they use the CUDA runtime the application already links.
namespace pppm_compat {

inline bool BiotSavartSolver::ensure_u(uint m) {
    if (m > capU_) {
        for (int c = 0; c < 3; c++) {
            cudaFree(U_[c]);
            U_[c] = nullptr;
            u_arr_[c] = GpuArrayd();
        }
        capU_ = 0;
        for (int c = 0; c < 3; c++)
            if (cudaMalloc(&U_[c], sizeof(double) * (m ? m : 1)) != cudaSuccess) return false;
        capU_ = m;
    }
    for (int c = 0; c < 3; c++) u_arr_[c] = GpuArrayd(U_[c], m);
    return true;
}

inline bool BiotSavartSolver::refresh_sorted() {
    if (sorted_valid_) return true;
    if (N_ > capS_) {
        cudaFree(spos_);
        spos_ = nullptr;
        for (int c = 0; c < 3; c++) { cudaFree(salpha_[c]); salpha_[c] = nullptr; }
        capS_ = 0;
        if (cudaMalloc(&spos_, sizeof(float4) * N_) != cudaSuccess) return false;
        for (int c = 0; c < 3; c++)
            if (cudaMalloc(&salpha_[c], sizeof(double) * N_) != cudaSuccess) return false;
        capS_ = N_;
    }
    sorted_valid_ = pppm_get_sorted_vortices(scene_, reinterpret_cast<float *>(spos_), salpha_[0], salpha_[1],
                                             salpha_[2]) == PPPM_OK;
    spos_arr_ = GpuArrayf4(spos_, N_);
    for (int c = 0; c < 3; c++) salpha_arr_[c] = GpuArrayd(salpha_[c], N_);
    return sorted_valid_;
}

inline void BiotSavartSolver::free_buffers() {
    for (int c = 0; c < 3; c++) {
        cudaFree(U_[c]);
        U_[c] = nullptr;
        cudaFree(salpha_[c]);
        salpha_[c] = nullptr;
    }
    cudaFree(spos_);
    spos_ = nullptr;
    capU_ = capS_ = 0;
    for (int c = 0; c < 3; c++) u_arr_[c] = salpha_arr_[c] = GpuArrayd();
    spos_arr_ = GpuArrayf4();
    sorted_valid_ = false;
}

}  // namespace pppm_compat

inline bool pppm_compat::PotentialFieldSolver::ensure_out(uint m) {
    if (m <= cap_) return true;
    cudaFree(grad_);
    cudaFree(dphidn_);
    cudaFree(split_);
    grad_ = nullptr;
    dphidn_ = nullptr;
    split_ = nullptr;
    const size_t k = m ? m : 1;
    if (cudaMalloc(&grad_, sizeof(double3) * k) != cudaSuccess) return false;
    if (cudaMalloc(&dphidn_, sizeof(double) * k) != cudaSuccess) return false;
    if (cudaMalloc(&split_, sizeof(double) * 6 * k) != cudaSuccess) return false;
    cap_ = m;
    return true;
}

inline bool pppm_compat::PotentialFieldSolver::computeDphiDn() {
    // de-interleave normals and gradients with strided 2-D copies, then the
    // library's element-wise kernel
    const size_t k = cap_ ? cap_ : 1;
    double *dst[6] = {split_, split_ + k, split_ + 2 * k, split_ + 3 * k, split_ + 4 * k, split_ + 5 * k};
    const double *n = reinterpret_cast<const double *>(normals_);
    const double *g = reinterpret_cast<const double *>(grad_);
    const double *src[6] = {n, n + 1, n + 2, g, g + 1, g + 2};
    for (int c = 0; c < 6; c++)
        if (cudaMemcpy2D(dst[c], sizeof(double), src[c], 3 * sizeof(double), sizeof(double), M_,
                         cudaMemcpyDeviceToDevice) != cudaSuccess)
            return false;
    return pppm_potential_dphidn(p_, M_, dst[0], dst[1], dst[2], dst[3], dst[4], dst[5], mass_, areas_, dphidn_) ==
           PPPM_OK;
}

inline bool pppm_compat::PotentialFieldSolver::shutdown() {
    if (p_) pppm_potential_destroy(p_);
    p_ = nullptr;
    cudaFree(grad_);
    cudaFree(dphidn_);
    cudaFree(split_);
    grad_ = nullptr;
    dphidn_ = nullptr;
    split_ = nullptr;
    cap_ = 0;
    return true;
}
