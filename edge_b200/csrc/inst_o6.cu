// Compiled configurations of order 6 (precision, fused runs, relaxation mechanisms: inst_o6.inc),
// one of four parts per object (inst_order.cuh).
#define EDGE_B200_ORDER 6
#define EDGE_B200_INC "inst_o6.inc"
#include "inst_order.cuh"
