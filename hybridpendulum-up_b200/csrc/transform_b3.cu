// Synthesis and analysis launchers (transform_b.cuh) for the bandlimits
// B = 3, 7, 11, 15, 19, 23, 27, 31 (B mod 4 = 3).
#define HP_TRANSFORM_PART 3
#include "transform_b.cuh"

HP_INST_B(3)
HP_INST_B(7)
HP_INST_B(11)
HP_INST_B(15)
HP_INST_B(19)
HP_INST_B(23)
HP_INST_B(27)
HP_INST_B(31)
