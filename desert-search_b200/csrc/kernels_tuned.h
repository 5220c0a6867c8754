// Launch shapes of the table, flood-evaluation and proxy-zone kernels, as chosen by
// desert-search_b200/tune_kernels.py on a B200 (each candidate built with -D overrides, its outputs checked
// bit for bit against the default build, timed on fixed work).  A -D on the compiler command line overrides them.
#pragma once
#ifndef DSG_TAB_WAVES
#define DSG_TAB_WAVES 4         // k_tables: the fewest bands per table (1-8) giving at least this many waves of CTAs
#endif
#ifndef DSG_EVAL_RUN
#define DSG_EVAL_RUN 16         // k_tile_eval: most consecutive sub-blocks a block takes from the round queue at once
#endif
#ifndef DSG_EVAL_BLOCKS
#define DSG_EVAL_BLOCKS 0       // k_tile_eval: blocks per SM in a round's grid (0 = the occupancy limit)
#endif
#ifndef DSG_EVAL_MINB
#define DSG_EVAL_MINB 4         // k_tile_eval: resident blocks per SM its register budget is cut for
#endif
#ifndef DSG_PROXY_MINB
#define DSG_PROXY_MINB 4        // k_proxy: resident blocks per SM its register budget is cut for (1: no cut)
#endif
#ifndef DSG_ZONE_CHUNK
#define DSG_ZONE_CHUNK 2048     // proxy zone kernels: cells per block step
#endif
