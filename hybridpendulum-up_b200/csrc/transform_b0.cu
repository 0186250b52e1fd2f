// Synthesis and analysis launchers (transform_b.cuh) for the bandlimits
// B = 4, 8, 12, 16, 20, 24, 28, 32 (B mod 4 = 0).
#define HP_TRANSFORM_PART 0
#include "transform_b.cuh"

HP_INST_B(4)
HP_INST_B(8)
HP_INST_B(12)
HP_INST_B(16)
HP_INST_B(20)
HP_INST_B(24)
HP_INST_B(28)
HP_INST_B(32)
