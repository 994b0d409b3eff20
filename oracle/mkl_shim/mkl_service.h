/*
 * Oracle infrastructure (test-only).  Stand-in for MKL's version query, which
 * the reference calls from MklFactory::display_info (MklFactory.cpp:89-100).
 */
#ifndef LFTS_ORACLE_MKL_SERVICE_SHIM_H_
#define LFTS_ORACLE_MKL_SERVICE_SHIM_H_

typedef struct {
    int MajorVersion;
    int MinorVersion;
    int UpdateVersion;
    const char *ProductStatus;
    const char *Build;
    const char *Processor;
    const char *Platform;
} MKLVersion;

#ifdef __cplusplus
extern "C" {
#endif
void mkl_get_version(MKLVersion *version);
#ifdef __cplusplus
}
#endif

#endif
