/*
 * Force-included (gcc -include) into every reference 2DCode translation unit built for
 * the oracle.  Three jobs, none of which changes the arithmetic:
 *
 *  1. exit() -> dgr_ref_exit(): the reference stops the process on a NaN flux or a
 *     negative depth (2DCode/compute2DL.c:245-302, 2DCode/wetDry2D.c:142-146,233-237).
 *     Inside a test process that would kill the test runner, so the oracle driver
 *     longjmp()s back to its caller and reports the failure as a status instead.
 *  2. printf() -> dgr_ref_printf(): keeps the per-step "dt = / time =" chatter of
 *     2DCode/time_evolution.c:314-315 off stdout and keeps the last message, which
 *     carries the failing edge or element index.
 *  3. junc->WD: under -DWDON 2DCode/compute2DL.c:203,251,270 read the wet/dry flags
 *     through a ChanNet junction pointer that 2DCode does not have.  The macro makes
 *     that expression read the 2DCode global WD (2DCode/MeshAttributes.h:42).
 */
#ifndef ORACLE_SHIM_REF_HOOKS_H
#define ORACLE_SHIM_REF_HOOKS_H

#include <stdio.h>
#include <stdlib.h>

void dgr_ref_exit(int status) __attribute__((noreturn));
int dgr_ref_printf(const char *fmt, ...);

#define exit dgr_ref_exit
#define printf dgr_ref_printf

extern int *WD;
#define junc (&(struct { int *WD; }){ WD })

#endif
