/*
 * ORACLE (test infrastructure only): drives the unmodified ChanNet/internal_BC.c — the
 * reference's channel <-> junction coupling — on caller-given arrays.  It builds the
 * reference's own `struct channel` / `struct junction` (ChanNet/ChannelsAndJunctions.h)
 * around the caller's buffers, with one junction, calls internal_BC() and leaves the
 * results in those buffers.  Same signature as orc_internal_bc in dgr_oracle.c.
 */
#include <stdlib.h>

#include "ChannelsAndJunctions.h"
#include "MeshAttributes.h"

extern void internal_BC(void);

const double g = 9.81;
int NumChannels;
int NumJunctions;
struct channel **ChannelList;
struct junction **JunctionList;

int ref_internal_bc(int ne, int nf, const double *x, const double *y, const double *z, const int *el2v,
                    const int *ed2v, const int *ed2el, const double *zeta, const double *qx, const double *qy,
                    double *bzeta, double *bqn, int nchan, const int *in_ptr, const int *in_edges,
                    const int *out_ptr, const int *out_edges, const int *chan_nodes, const int *chan_off,
                    double *A, double *Q)
{
    struct junction junc = {0};
    junc.TotalNumEdges = nf;
    junc.NumEl = ne;
    junc.x = (double *)x;
    junc.y = (double *)y;
    junc.z = (double *)z;
    junc.EltoVert = (int *)el2v;
    junc.EdgtoVert = (int *)ed2v;
    junc.EdgtoEls = (int *)ed2el;
    junc.zeta = (double *)zeta;
    junc.Qx = (double *)qx;
    junc.Qy = (double *)qy;
    junc.bzeta = bzeta;
    junc.bQn = bqn;
    struct junction *jl[1] = {&junc};
    struct channel *chans = calloc((size_t)(nchan ? nchan : 1), sizeof(struct channel));
    struct channel **cl = calloc((size_t)(nchan ? nchan : 1), sizeof(struct channel *));
    int *lists = calloc((size_t)2 * (in_ptr[nchan] + out_ptr[nchan]) + 2, sizeof(int));
    const int nodes = nchan ? chan_off[nchan - 1] + chan_nodes[nchan - 1] : 0;
    double *width = calloc((size_t)nodes + 1, sizeof(double)); /* read (not used) by internal_BC */
    if (!chans || !cl || !lists || !width) {
        free(chans);
        free(cl);
        free(lists);
        free(width);
        return -1;
    }
    int *p = lists;
    for (int ch = 0; ch < nchan; ++ch) {
        struct channel *c = chans + ch;
        c->NumNodes = chan_nodes[ch];
        c->NumEl = chan_nodes[ch] - 1;
        c->A = A + 2 * (size_t)chan_off[ch];
        c->Q = Q + 2 * (size_t)chan_off[ch];
        c->b = width + chan_off[ch];
        c->NumInflowJunctionEdges = in_ptr[ch + 1] - in_ptr[ch];
        c->InflowJunctionEdges = p;
        for (int j = in_ptr[ch]; j < in_ptr[ch + 1]; ++j) {
            *p++ = in_edges[j];
            *p++ = 0;
        }
        c->NumOutflowJunctionEdges = out_ptr[ch + 1] - out_ptr[ch];
        c->OutflowJunctionEdges = p;
        for (int j = out_ptr[ch]; j < out_ptr[ch + 1]; ++j) {
            *p++ = out_edges[j];
            *p++ = 0;
        }
        cl[ch] = c;
    }
    NumChannels = nchan;
    NumJunctions = 1;
    ChannelList = cl;
    JunctionList = jl;
    internal_BC();
    ChannelList = NULL;
    JunctionList = NULL;
    free(chans);
    free(cl);
    free(lists);
    free(width);
    return 0;
}
