// salmon_oracle_gs.cpp -- ground-state pieces of the CPU oracle (test
// infrastructure only).  Filled in with the CG eigensolver restatement.
#include "salmon_oracle.h"
