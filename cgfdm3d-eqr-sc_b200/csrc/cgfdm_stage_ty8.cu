// The fused CGFDM stage with 32 x 8 column tiles (two CTAs per SM), in
// namespace cgfdm::ty8: the same source as cgfdm_stage.cu, compiled for the
// other tile height.  Sessions of the FP32 split pipeline use it by default
// (measured 6 % faster per step on 400 x 400 x 200 than 32 x 4 tiles); the
// autotuner may choose either.
#define CG_TILE_Y 8
#define CG_CTAS_PER_SM 2
#define CG_TILE_NS ty8
#include "cgfdm_stage.cu"
