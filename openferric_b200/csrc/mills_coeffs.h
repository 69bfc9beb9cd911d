/* Generated by openferric_b200/csrc/fit_mills.py; do not edit by hand.
 * Mills ratio M(x) = (1 - Phi(x)) / phi(x) = t P(t), t = 1 / (1 + 0.4 x), x >= 0.
 * Max float32 relative error over x in [0, 13]: 3.908e-07 */
#pragma once
#define OF_MILLS_C 4.000000000e-01f
#define OF_MILLS_DEG 9
static __device__ __constant__ const float kMills[10] = {3.999999464e-01f, 4.000152946e-01f, 3.354167938e-01f, 2.165435702e-01f, -1.600099541e-02f, 1.723066866e-01f, -7.444626689e-01f, 7.827905416e-01f, -3.555635512e-01f, 6.226849183e-02f};
