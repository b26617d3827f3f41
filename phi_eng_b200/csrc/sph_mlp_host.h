// Internal bridge between the closure network object (sph_mlp.cu) and the
// world's closure step (sph_world.cu).
#pragma once

#include "phieng_sph.h"
#include "sph_mlp.cuh"

// Device view of a network's BF16 images, biases and normalisation.
phieng::MlpDev phieng_mlp_dev(const PhiengMlp* m);

namespace phieng {
// Training grid for a batch (multiple of 128): CTAs and 128-sample rounds per CTA.
void mlp_grid(uint32_t batch, uint32_t* ctas, uint32_t* rounds);
}  // namespace phieng
