// bm_internal.h — shared host/device definitions of the B200 MPM library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bm_mpm.h"

namespace bm {

// Device-side error bits, OR-ed into Solver::d_status[0].
enum : uint32_t { ERR_ESCAPE = 1u, ERR_NONFINITE = 2u };

// Particle planes of the SoA store (each plane holds `cap` floats).
enum Plane : int {
    P_X = 0,   // position x, y, z       (3)
    P_V = 3,   // velocity               (3)
    P_F = 6,   // deformation gradient   (9, row-major)
    P_C = 15,  // APIC affine matrix     (9, row-major)
    P_M = 24,  // mass                   (1)
    P_V0 = 25, // reference volume V0    (1)
    N_PLANES = 26
};

// Dense grid box, blocked in 4^3-node blocks aligned to absolute node
// indices (the reference's block grid, spgrid_cpu.h:93-105). Node (i,j,k)
// lives at block ((i-ox)>>2, (j-oy)>>2, (k-oz)>>2) and local slot
// (i&3)*16 + (j&3)*4 + (k&3).
struct GridDesc {
    int ox, oy, oz;       // origin node, multiple of 4
    int nbx, nby, nbz;    // blocks per axis
    float dx, inv_dx;
    __host__ __device__ int64_t num_blocks() const { return (int64_t)nbx * nby * nbz; }
    __host__ __device__ int64_t num_nodes() const { return num_blocks() * 64; }
    // Linear node index, or -1 outside the box.
    __host__ __device__ __forceinline__ int64_t node(int i, int j, int k) const {
        const int ri = i - ox, rj = j - oy, rk = k - oz;
        if ((unsigned)ri >= (unsigned)(nbx * 4) || (unsigned)rj >= (unsigned)(nby * 4) ||
            (unsigned)rk >= (unsigned)(nbz * 4))
            return -1;
        const int64_t b = ((int64_t)(ri >> 2) * nby + (rj >> 2)) * nbz + (rk >> 2);
        return b * 64 + ((ri & 3) * 16 + (rj & 3) * 4 + (rk & 3));
    }
};

// Material and integration constants, derived on the host in float exactly
// like mpm_solver.h:111-112 and :149-151.
struct Material {
    float mu, lambda;
    float neg_alpha_koh;  // (-alpha) * (3 lambda + 2 mu) / (2 mu)
    float floor_friction;
    float gx, gy, gz;
};

struct ParticleSoA {
    float* base;   // N_PLANES planes of `cap` floats
    int64_t cap;
    int64_t n;
    __host__ __device__ __forceinline__ float* plane(int p) const { return base + (int64_t)p * cap; }
};

struct GridBuffers {
    float4* mv;      // momentum (after update: velocity) xyz, mass w
    float4* f;       // force xyz
    uint8_t* alloc;  // per block: ever touched
};

// Kernel launchers (bm_step_kernels.cu, bm_m1.cu).
void launch_p2g(const ParticleSoA& ps, const GridDesc& g, const GridBuffers& gb, const Material& mat, float dt,
                uint32_t* d_status, unsigned long long* d_escaped, cudaStream_t st);
void launch_grid_update(const GridDesc& g, const GridBuffers& gb, const Material& mat, float dt, cudaStream_t st);
void launch_g2p(const ParticleSoA& ps, const GridDesc& g, const GridBuffers& gb, const Material& mat, float dt,
                uint32_t* d_status, unsigned long long* d_escaped, cudaStream_t st);

// M1 PIC-rigid coupler; accumulates into d_acc (6 doubles + 1 count as double).
struct M1Params {
    float R[9];          // body-to-world rotation, row-major (host float, no FMA)
    float c[3], vl[3], w[3];
    float he[3];
    float lo[3], hi[3];  // world AABB of the box formula
    float mb;            // per-node body mass
    float mb_over_dt;
    int shape;
    int bi0, bj0, bk0, nbi, nbj, nbk;  // candidate block range (relative to box)
};
bool m1_prepare(const GridDesc& g, const bm_collider_t& b, float dt, M1Params* out);
void launch_m1(const GridDesc& g, const GridBuffers& gb, const M1Params& p, double* d_acc, cudaStream_t st);
void launch_reaction_finalize(const double* d_acc, int n_bodies, bm_reaction_t* d_out, cudaStream_t st);

// Dense (i,j,k) copies between the blocked device layout and host order.
void launch_grid_to_dense(const GridDesc& g, const GridBuffers& gb, float* vel, float* force, float* mass,
                          uint8_t* active, uint8_t* balloc, cudaStream_t st);
void launch_dense_velocity_to_grid(const GridDesc& g, const GridBuffers& gb, const float* vel, cudaStream_t st);
void launch_seed_grid(const GridDesc& g, const GridBuffers& gb, int64_t n, const int32_t* ijk, const float* vel,
                      const float* mass, uint32_t* d_status, cudaStream_t st);

// Thread-local error text.
void set_last_error(const std::string& s);

}  // namespace bm
