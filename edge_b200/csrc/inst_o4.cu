// Compiled configurations of order 4 (precision, fused runs, relaxation mechanisms: inst_o4.inc),
// one of four parts per object (inst_order.cuh).
#define EDGE_B200_ORDER 4
#define EDGE_B200_INC "inst_o4.inc"
#include "inst_order.cuh"
