// terrain_f32.cu -- the FP32 (mixed-form) instantiations of the terrain
// passes, compiled beside terrain.cu so that the two halves build side by side.
#define ERFB_TER_F32 1
#include "terrain.cu"
