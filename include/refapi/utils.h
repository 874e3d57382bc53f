/*
 * utils.h -- FOR-QAOA's timing globals (include/utils.h:17-37 of the
 * reference): wall-clock start/end/diff (microseconds) and millisecond
 * accumulators the `weighted` driver prints.
 */
#ifndef FQ_REFAPI_UTILS_H_
#define FQ_REFAPI_UTILS_H_

#include <sys/time.h>

extern struct timeval start;
extern struct timeval end_;
extern unsigned long diff;

extern float rx_gate_time_ms;
extern float csqs_time_ms;
extern float transmission_time_ms;

#define MEASURET_START                  \
    do {                                \
        gettimeofday(&start, NULL);     \
    } while (0)

#define MEASURET_END                                                                  \
    do {                                                                              \
        gettimeofday(&end_, NULL);                                                    \
        diff += 1000000 * (end_.tv_sec - start.tv_sec) + end_.tv_usec - start.tv_usec; \
    } while (0)

#endif
