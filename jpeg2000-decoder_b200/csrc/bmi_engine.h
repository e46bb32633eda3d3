/*
 * bmi_engine.h — internal hooks between the BMI decoder front ends and the GPU engine
 * that are not part of the public C ABI.
 */
#pragma once
#include "../../include/j2k_gpu.h"

namespace bmi_engine {
/* Reference DecodeJobConfig::mCheckOutComponent: for RGB outputs write only component
 * `comp` (after the inverse MCT) into R, G and B; -1 = all components. */
int set_checkout(j2k_gpu_ctx *ctx, int slot, int comp);
}  // namespace bmi_engine
