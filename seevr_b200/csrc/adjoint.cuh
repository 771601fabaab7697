// adjoint.cuh — reverse mode of one substep (adjoint.cu).
#pragma once
#include "common.cuh"

namespace seevr {

// Gradient buffers (device), indexed like the body / geom arrays.
struct Grads {
    float* pos;       // [N*3]  in: dL/d pos after the substep, out: before
    float* quat;      // [N*4]
    float* vel;       // [N*3]
    float* omega;     // [N*3]
    float* friction;  // [G]    accumulated: dL/d geom_friction
};

// Adjoint work arrays (device).
struct AdjScratch {
    float* tape;     // [max_contacts * iterations * 13] inputs of every contact update
    uint4* ptape;    // [max_pairs * 2] supporting hull vertices per pair
    uint4* ctape;    // [max_contacts * 2] ... per contact
    float* vw;       // [N*6] velocities during the recomputed sweep
    float* gv;       // [N*3] running dL/dv
    float* gw;       // [N*3] running dL/dω
    float* gR;       // [N*9] dL/dR (rotation matrix, by columns)
    float* gp;       // [N*3] dL/d position
    float* gq;       // [N*4] dL/d quaternion
    float* gc;       // [max_contacts*12] dL/d (n, ra, rb, bias, kn, mu) per contact
    float* glam;     // [max_contacts] dL/dλ
    float* lam;      // [max_contacts] λ during the recomputed sweep
    float* par;      // [max_contacts*12] contact constants (n, ra, rb, bias, kn, mu)
};

int launch_adjoint(const World& w, const Consts& k, const Scratch& s, const AdjScratch& a,
                   const Grads& g, float dt, cudaStream_t st);

}  // namespace seevr
