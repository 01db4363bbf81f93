// Compiled configurations of order 2 (precision, fused runs, relaxation mechanisms: inst_o2.inc),
// one of four parts per object (inst_order.cuh).
#define EDGE_B200_ORDER 2
#define EDGE_B200_INC "inst_o2.inc"
#include "inst_order.cuh"
