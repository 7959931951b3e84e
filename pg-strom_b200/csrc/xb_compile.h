/*
 * xb_compile.h - OpenSession-time bytecode translator (xb_compile.cpp)
 */
#ifndef XB_COMPILE_H
#define XB_COMPILE_H
#include <stddef.h>
#include <stdint.h>
#include "xb_plan.h"

#ifdef __cplusplus
extern "C" {
#endif
/*
 * Validates every kern_expression of the session and lowers it into the
 * register program of *plan.  dev_session_base is the device address the
 * session blob is copied to (constants are referenced in place).
 * Returns 0 on success, -1 with a message in errmsg otherwise.
 */
int xb_compile_session(const kern_session_info *session, size_t session_sz,
                       uint64_t dev_session_base,
                       const kern_multirels *kmrels,
                       xb_plan *plan, char *errmsg, size_t errlen);
#ifdef __cplusplus
}
#endif
#endif
