// contact.h -- the step with the CT-Contact EMF (contact.cu).
#pragma once

#include <cuda_runtime.h>

#include "rmhd2d_internal.h"

namespace rmhd2d {

struct ContactStep {
    Grid g;
    double *A;            // U^n in, U^{n+1} out (8 planes)
    double *B;            // U* (8 planes)
    double *C;            // the stage-2 result before CT (8 planes)
    double *F1, *G1;      // stage-1 fluxes (8 planes each)
    double *F2, *G2;      // stage-2 fluxes (8 planes each)
    double *R1, *R2;      // per-cell reference EMFs of the two stages (1 plane each)
    double *E;            // corner EMFs, the mean of the two stages' (1 plane)
    const double *eta;    // eta plane or nullptr
    double *row2;         // the symmetric-wall boundary's row buffer
    Control *ctl;
    int parity;
};

void enqueue_contact_step(const ContactStep &c, cudaStream_t st);

}  // namespace rmhd2d
