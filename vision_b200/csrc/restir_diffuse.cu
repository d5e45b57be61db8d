// The ReSTIR kernels of restir.cu compiled for scenes whose surfaces are
// diffuse or emitters (black body) only.
#include "vs_scene.h"

#define VS_RT_MATERIALS ((1u << vs::kMatDiffuse) | (1u << vs::kMatBlackBody))
#define VS_RT_NS rt_diffuse
// 5 blocks of 128 for the light candidates (96 registers, 88 bytes of
// spills) measured 1.6 % faster per many-light frame than 4 (128 registers).
#define VS_RT_LIGHTS_MIN_BLOCKS 5
#include "restir.cu"
