/* Generated by openferric_b200/csrc/fit_invnorm.py; do not edit by hand.
 * Phi^-1(u) = x * P(w), x = 2u-1, w = -log2(4u(1-u)); central P in (w - 3.625) for w < 7.25,
 * tail P in (sqrt(w) - 3.895800959).  Max float32 relative error on u = (k+0.5) 2^-23: 2.995e-07 */
#pragma once
#define OF_INVN_W_SPLIT 7.250000000e+00f
#define OF_INVN_C_CENTER 3.625000000e+00f
#define OF_INVN_T_CENTER 3.895800959e+00f
#define OF_INVN_DEG_C 8
#define OF_INVN_DEG_T 8
static __device__ __constant__ const float kInvnCentral[9] = {2.127727985e+00f, 2.416673601e-01f, -2.870769473e-03f, -5.852763425e-04f, 7.125214324e-05f, -1.050068590e-06f, -5.462189847e-07f, 3.742659871e-08f, 2.041509406e-09f};
static __device__ __constant__ const float kInvnTail[9] = {4.351985455e+00f, 1.183515310e+00f, 5.344662815e-03f, -3.082651645e-03f, 1.698795008e-03f, -1.056959736e-03f, 5.093832733e-04f, -6.714181654e-05f, -3.130684854e-05f};
