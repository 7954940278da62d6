// rs_host.h -- internal helpers shared by the host services and the engine.
#pragma once
#include "rssieve_b200.h"

#ifdef __cplusplus
extern "C" {
#endif
// record a printf-style message for rs_last_error() on this thread
void rs_set_error(const char *fmt, ...);
// structural checks of a job (base, counts, k, c, n-range, bitmap size)
int rs_seqs_validate(const rs_seqs *s);
#ifdef __cplusplus
}
#endif
