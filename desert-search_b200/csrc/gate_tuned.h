// Launch shapes of the gate kernels, as chosen by desert-search_b200/tune_gate.py on a B200 (each candidate
// built, checked bit for bit against the default build, and timed with dsg_gate_bench).  A -D on the
// compiler command line overrides them; that is how the tuner builds its candidates.
#pragma once
#ifndef DSG_PG_MINBLOCKS
#define DSG_PG_MINBLOCKS 6      // k_pregate blocks per SM (register cap 65536 / (64 x this))
#endif
#ifndef DSG_FG_MINBLOCKS
#define DSG_FG_MINBLOCKS 4      // k_fullgate blocks per SM (register cap 65536 / (128 x this))
#endif
#ifndef DSG_FG_ROWS
#define DSG_FG_ROWS 8           // k_fullgate rows staged in shared memory per block step
#endif
