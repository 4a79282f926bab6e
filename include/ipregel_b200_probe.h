/*
 * ipregel_b200_probe.h -- measurement library of the benchmark, kept apart
 * from the runtime (libipregel_b200.so): lib/libipregel_b200_probe.so.  The
 * engine never calls it; bench.py reports its rates beside the kernels' own.
 */
#ifndef IPREGEL_B200_PROBE_H
#define IPREGEL_B200_PROBE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The random-gather ceiling -- no counterpart in the reference.  Times n
 * reads of `row_bytes`-byte rows (4; or 64, 128, 256 read as 16-byte quads
 * by 4, 8, 16 consecutive threads) at pseudo-random positions of a table of `table_bytes`, each
 * position taken from a coalesced u32 index stream: the access pattern of
 * the push prechecks and of the pull gathers, with nothing else.  Returns
 * rows read per second and (index + row) bytes per second in GB/s, averaged
 * over `reps` launches after one warm-up launch.  Allocates n * 4 +
 * table_bytes of device memory for the call; synchronous. */
int ipg_measure_gather(uint64_t table_bytes, uint32_t row_bytes, uint64_t n, int reps, double* rows_per_s,
                       double* gbs);

/* Message of the calling thread's last failed probe call. */
const char* ipg_probe_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* IPREGEL_B200_PROBE_H */
