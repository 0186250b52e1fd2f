// Synthesis and analysis launchers (transform_b.cuh) for the bandlimits
// B = 2, 6, 10, 14, 18, 22, 26, 30 (B mod 4 = 2).
#define HP_TRANSFORM_PART 2
#include "transform_b.cuh"

HP_INST_B(2)
HP_INST_B(6)
HP_INST_B(10)
HP_INST_B(14)
HP_INST_B(18)
HP_INST_B(22)
HP_INST_B(26)
HP_INST_B(30)
