/*
 * One reference evaluation context (test infrastructure): the reference's
 * own par/mod/dat structs (src/shape/shape2.h), filled by ref_harness.c.
 */
#ifndef REF_SESSION_H
#define REF_SESSION_H

typedef struct ref_session {
    struct par_t par;
    struct mod_t mod;
    struct dat_t dat;
    int nsets_cap;
} ref_session;

#endif
