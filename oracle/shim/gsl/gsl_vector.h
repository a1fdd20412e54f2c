/*
 * Stand-in for the few GSL dense-vector calls that 2DCode/time_evolution.c:14-243
 * makes (alloc, free, set, get, scale, add, fprintf).  Written for the oracle build
 * of the reference only; GSL itself is not installed here.
 *
 * Every element operation is one IEEE double multiply (scale) or add (add), which is
 * all GSL's own vector routines do for unit-stride vectors, so the reference step
 * gives the same bits with this header as with GSL.
 */
#ifndef ORACLE_SHIM_GSL_VECTOR_H
#define ORACLE_SHIM_GSL_VECTOR_H

#include <stdio.h>
#include <stdlib.h>

typedef struct {
    size_t size;
    double *data;
} gsl_vector;

static inline gsl_vector *gsl_vector_alloc(size_t n)
{
    gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
    if (!v) return NULL;
    v->size = n;
    v->data = (double *)malloc((n ? n : 1) * sizeof(double));
    return v;
}

static inline void gsl_vector_free(gsl_vector *v)
{
    if (!v) return;
    free(v->data);
    free(v);
}

static inline void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i] = x; }
static inline double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i]; }

static inline int gsl_vector_scale(gsl_vector *v, double x)
{
    for (size_t i = 0; i < v->size; ++i) v->data[i] *= x;
    return 0;
}

static inline int gsl_vector_add(gsl_vector *a, const gsl_vector *b)
{
    for (size_t i = 0; i < a->size; ++i) a->data[i] += b->data[i];
    return 0;
}

static inline int gsl_vector_fprintf(FILE *f, const gsl_vector *v, const char *fmt)
{
    for (size_t i = 0; i < v->size; ++i) {
        fprintf(f, fmt, v->data[i]);
        fputc('\n', f);
    }
    return 0;
}

#endif
