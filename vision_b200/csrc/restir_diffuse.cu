// The ReSTIR kernels of restir.cu compiled for scenes whose surfaces are
// diffuse or emitters (black body) only.
#include "vs_scene.h"

#define VS_RT_MATERIALS ((1u << vs::kMatDiffuse) | (1u << vs::kMatBlackBody))
#define VS_RT_NS rt_diffuse
#include "restir.cu"
