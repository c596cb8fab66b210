/* ufsecp_error.h -- error codes shared by the verify ABI.
 *
 * Values are those of the reference's include/ufsecp/ufsecp_error.h:23-36 so
 * that callers' error handling keeps working: 0 = success, CPU-style codes
 * 1..13, GPU codes 100..106 (declared in ufsecp_gpu.h). */
#ifndef UFSECP_ERROR_H
#define UFSECP_ERROR_H

#include "ufsecp_version.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int ufsecp_error_t;

#define UFSECP_OK                 0
#define UFSECP_ERR_NULL_ARG       1
#define UFSECP_ERR_BAD_KEY        2
#define UFSECP_ERR_BAD_PUBKEY     3
#define UFSECP_ERR_BAD_SIG        4
#define UFSECP_ERR_BAD_INPUT      5
#define UFSECP_ERR_VERIFY_FAIL    6
#define UFSECP_ERR_ARITH          7
#define UFSECP_ERR_SELFTEST       8
#define UFSECP_ERR_INTERNAL       9
#define UFSECP_ERR_BUF_TOO_SMALL  10
#define UFSECP_ERR_NOT_FOUND      11
#define UFSECP_ERR_DEPRECATED_API 12
#define UFSECP_ERR_CANCELLED      13

#ifdef __cplusplus
}
#endif

#endif /* UFSECP_ERROR_H */
