// adjoint.cuh — reverse mode of one substep (adjoint.cu).
#pragma once
#include "common.cuh"

namespace seevr {

// Gradient buffers (device, FP64), indexed like the body / geom arrays.
struct Grads {
    double* pos;       // [N*3]  in: dL/d pos after the substep, out: before
    double* quat;      // [N*4]
    double* vel;       // [N*3]
    double* omega;     // [N*3]
    double* friction;  // [G]    accumulated: dL/d geom_friction
};

// Adjoint work arrays (device).
struct AdjScratch {
    float* tape;     // [max_contacts * iterations * 13] inputs of every contact update
    uint4* ptape;    // [max_pairs * 2] supporting hull vertices per pair
    uint4* ctape;    // [max_contacts * 2] ... per contact
    float* vw;       // [N*6] velocities during the recomputed sweep
    // reverse-pass accumulators, FP64
    double* gv;      // [N*3] running dL/dv
    double* gw;      // [N*3] running dL/dω
    double* gR;      // [N*9] dL/dR (rotation matrix, by columns)
    double* gp;      // [N*3] dL/d position
    double* gq;      // [N*4] dL/d quaternion
    double* gc;      // [max_contacts*12] dL/d (n, ra, rb, bias, kn, mu) per contact
    double* glam;    // [max_contacts] dL/dλ
    float* lam;      // [max_contacts] λ during the recomputed sweep
    float* par;      // [max_contacts*12] contact constants (n, ra, rb, bias, kn, mu)
    // wavefront levels of each bundle's contacts
    uint32_t* last;  // [N] latest level per body
    uint32_t* level; // [max_contacts]
    uint32_t* order; // [max_contacts] contacts grouped by level
    uint32_t* lvl;   // [max_contacts + max_scenes + 2] level boundaries per bundle
    // contributions to fixed bodies' gradients, per contact and side (summed
    // in contact order at the end): v3 w3 p3 R9 friction1 (stride 20)
    double* fix;     // [max_contacts*40]
};

int launch_adjoint(const World& w, const Consts& k, const Scratch& s, const AdjScratch& a,
                   const Grads& g, float dt, cudaStream_t st);

}  // namespace seevr
