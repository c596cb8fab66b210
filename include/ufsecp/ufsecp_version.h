/* ufsecp_version.h -- export macro and version of the B200 verify library.
 *
 * Same role and macro names as the reference's include/ufsecp/ufsecp_version.h
 * (UFSECP_API visibility macro), so code written against the reference's GPU
 * header compiles unchanged against this one.  The version numbers are this
 * library's; the ABI version matches the reference's (4) because the exported
 * signatures are the same. */
#ifndef UFSECP_VERSION_H
#define UFSECP_VERSION_H

#define UFSECP_VERSION_MAJOR 4
#define UFSECP_VERSION_MINOR 5
#define UFSECP_VERSION_PATCH 0
#define UFSECP_VERSION_STRING "4.5.0-b200"
#define UFSECP_ABI_VERSION 4

#ifndef UFSECP_API
#  if defined(__GNUC__) && __GNUC__ >= 4
#    define UFSECP_API __attribute__((visibility("default")))
#  else
#    define UFSECP_API
#  endif
#endif

#endif /* UFSECP_VERSION_H */
