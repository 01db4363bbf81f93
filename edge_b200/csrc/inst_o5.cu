// Compiled configurations of order 5 (precision, fused runs, relaxation mechanisms: inst_o5.inc),
// one of four parts per object (inst_order.cuh).
#define EDGE_B200_ORDER 5
#define EDGE_B200_INC "inst_o5.inc"
#include "inst_order.cuh"
