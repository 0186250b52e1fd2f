// Synthesis and analysis launchers (transform_b.cuh) for the bandlimits
// B = 5, 9, 13, 17, 21, 25, 29 (B mod 4 = 1).
#define HP_TRANSFORM_PART 1
#include "transform_b.cuh"

HP_INST_B(5)
HP_INST_B(9)
HP_INST_B(13)
HP_INST_B(17)
HP_INST_B(21)
HP_INST_B(25)
HP_INST_B(29)
