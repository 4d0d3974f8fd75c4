// sb200_gs.cuh -- ground-state helpers shared inside sb200_gs.cu.
#pragma once

#define TRY_GS(x)                     \
  do {                                \
    int _r = (x);                     \
    if (_r != SB200_OK) return _r;    \
  } while (0)
