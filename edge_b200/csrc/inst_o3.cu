// Compiled configurations of order 3 (precision, fused runs, relaxation mechanisms: inst_o3.inc),
// one of four parts per object (inst_order.cuh).
#define EDGE_B200_ORDER 3
#define EDGE_B200_INC "inst_o3.inc"
#include "inst_order.cuh"
