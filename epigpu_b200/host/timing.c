/*
 * timing.c -- wall-clock helpers for the host program (the role of src/timing.c):
 * a monotonic clock instead of time(NULL), and the "h hours, m minutes, s seconds"
 * format of readtime (src/timing.c:38-56).
 */
#include <math.h>
#include <stdio.h>
#include <time.h>

#include "epigpu_host.h"

double wall_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

void format_duration(char *out, size_t outlen, double s)
{
    if (s > 3600) {
        const double h = floor(s / 3600), m = floor((s - h * 3600) / 60);
        snprintf(out, outlen, "%0.0f hours, %0.0f minutes, %0.0f seconds", h, m, s - h * 3600 - m * 60);
    } else if (s > 60) {
        const double m = floor(s / 60);
        snprintf(out, outlen, "%0.0f minutes, %0.0f seconds", m, s - m * 60);
    } else {
        snprintf(out, outlen, "%0.3f seconds", s);
    }
}
