/* Compatibility header carrying the reference's header name (timing.h): the
 * monotonic tick counter that the reference's CLI and perf drivers print
 * their wall-clock times with (reference include/timing.h, src/timing.c),
 * provided by libgli_b200 so that those drivers link against it unchanged. */
#ifndef GLI_B200_COMPAT_TIMING_H
#define GLI_B200_COMPAT_TIMING_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* current time in ticks of a monotonic clock */
int64_t get_time_ticks(void);
/* ticks per second */
int64_t get_tick_resolution(void);

#ifdef __cplusplus
}
#endif
#endif
