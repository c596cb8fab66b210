/* ufsecp_cancel.h -- caller-driven cancellation token.
 *
 * The same type, layout and meaning as the reference's
 * include/ufsecp/ufsecp_cancel.h (UltrafastSecp256k1 v4.5.0), so that a token
 * built for the reference's long-running batch calls can be handed to this
 * library unchanged: a predicate the library polls between pieces of work,
 * the opaque pointer it is given back, and how many items may pass between two
 * polls (0 = the library's own piece size).  A NULL token, or a NULL
 * predicate, never cancels.  A non-zero answer ends the operation fail-closed
 * with UFSECP_ERR_CANCELLED: a cancelled request never reports verdicts, its
 * result bytes are cleared.  Cancellation is a status of the execution, not a
 * verdict.  Used here by ufsecp_gpu_ext_server_submit_cancellable. */
#ifndef UFSECP_CANCEL_H
#define UFSECP_CANCEL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Returns non-zero to ask for cancellation; `user` is the token's pointer. */
typedef int (*ufsecp_cancel_fn)(const void* user);

typedef struct ufsecp_cancel_token {
    ufsecp_cancel_fn is_cancelled;   /* NULL: never cancelled */
    const void* user;                /* passed back to is_cancelled, never dereferenced */
    uint32_t check_interval;         /* items between polls; 0: the library's default */
} ufsecp_cancel_token;

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
#define UFSECP_CANCEL_DEFAULT = nullptr
#else
#define UFSECP_CANCEL_DEFAULT
#endif

#endif /* UFSECP_CANCEL_H */
