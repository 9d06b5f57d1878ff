// bm_solver_impl.h — the plain solver handle (bm_solver_t) and its phase
// helpers, shared by the solver C ABI (bm_solver.cu) and the differentiable
// run built on it (bm_adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "bm_world.h"

struct bm_solver {
    bm::World w;
    bool acc_valid = false;           // acc[cur] holds P2G of the current particle state
    bool folded[2] = {false, false};  // acc[b].mv holds momentum + force * fold_dt[b]
    float fold_dt[2] = {0.0f, 0.0f};
    int view = 0;                     // buffer holding the grid a caller sees
    int32_t sort_interval = 32;  // the fused kernel's time measured the same at 8, 16 and 32
    int64_t steps_since_sort = 0;
    bool sorted = false;
    bool fast_math = false;
    int variant = 7;  // 128 threads x 7 CTAs per SM (72 registers): fastest on the 2M-particle wheel rut
    // couplers
    double* d_acc = nullptr;
    bm_reaction_t* d_react = nullptr;
    bm::M1Params* d_params = nullptr;
    double* d_frac_sum = nullptr;  // per body: the M4.5a overlap-fraction sum
    int react_cap = 0;
    int32_t coupler = BM_COUPLER_M1;  // coupler of bm_solver_step_coupled
    std::vector<bm::M1Params> h_params;

    bm::SceneHost& sc() { return w.scenes[0]; }
};

namespace bm {
namespace sol {

// Makes `dev` current for the lifetime of the guard.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Grid box and device scene table up to date (allocates on first use).
bm_status_t prepare(bm_solver* s);
// Sets the scene's dt (read by the kernels from the scene table).
void set_dt(bm_solver* s, float dt);
// grid.clear() + the standalone P2G of the current particle state.
bm_status_t do_p2g(bm_solver* s);
// update_grid on acc[cur] (unfolds a folded P2G of another dt first).
bm_status_t do_grid_update(bm_solver* s, float dt);
// M1 for each body in order on acc[cur]; reactions into s->d_react.
bm_status_t do_m1(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt);
// M0 for each body in order on acc[cur]; reactions into s->d_react.
bm_status_t do_m0(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt);
// The sweep coupler of layer 0 = M4.5a, 1 = M4.5b, 2 = M4.5 for each body in
// order on acc[cur]; reactions into s->d_react.
bm_status_t do_m45(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt, int layer);
// The standalone G2P from acc[cur].
bm_status_t do_g2p(bm_solver* s, float dt);
// The particle order or grid contents changed behind the solver's back.
void invalidate_state(bm_solver* s);

}  // namespace sol
}  // namespace bm
