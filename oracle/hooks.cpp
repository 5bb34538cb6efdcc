/*
 * oracle/hooks.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Linked into the same shared object as the reference's verbatim drivers
 * (drivers/sort-sources.cpp, drivers/upward.cpp, drivers/treecode-*.cpp), so it can
 * reach the driver's hidden globals.  It exports a few C entry points that let the
 * tests read what the reference computes inside one call:
 *   oracle_sort_sources  -> drivers/sort-sources.cpp:23-132 (keys, sorted x/y/v, bbox)
 *   oracle_tree_build    -> drivers/upward.cpp:280-314 (Tree::build) followed by a raw
 *                           dump of every node (s, e, childbase, innernode byte, mass,
 *                           com, radius, expansions) and Tree::dispose.
 *   oracle_order         -> the compile-time expansion order of this library.
 */
#include <cstring>
#include <cstdlib>

typedef REAL realtype;

#include "upward.h"
#include "sort-sources.h"

namespace Tree
{
    extern int currnnodes;
    extern realtype ext, xmin, ymin;
}

extern "C" __attribute__((visibility("default")))
int oracle_order(void) { return ORDER; }

extern "C" __attribute__((visibility("default")))
void oracle_sort_sources(const double *xsrc, const double *ysrc, const double *vsrc, int nsrc,
                         int *keys, double *xs, double *ys, double *vs, double *bbox3)
{
    sort_sources(xsrc, ysrc, vsrc, nsrc, keys, xs, ys, vs, bbox3 + 0, bbox3 + 1, bbox3 + 2);
}

/* Builds the reference tree and copies it out.  Returns the node count, or -(count)
 * when the caller's capacity is too small (nothing is copied then).  bbox3 gets
 * (xmin, ymin, ext); xs/ys/vs get the sorted sources (nsrc each). */
extern "C" __attribute__((visibility("default")))
int oracle_tree_build(const double *xsrc, const double *ysrc, const double *vsrc, int nsrc,
                      int leafcap, int capacity,
                      int *s, int *e, int *childbase, unsigned char *innernode,
                      double *mass, double *xcom, double *ycom, double *r, double *expansions,
                      double *xs, double *ys, double *vs, double *bbox3)
{
    Tree::build(xsrc, ysrc, vsrc, nsrc, leafcap);

    const int n = Tree::currnnodes;
    if (n > capacity) {
        Tree::dispose();
        return -n;
    }

    for (int i = 0; i < n; ++i) {
        const Tree::Node &nd = Tree::nodes[i];
        s[i] = nd.s;
        e[i] = nd.e;
        childbase[i] = nd.state.childbase;
        unsigned char b;
        std::memcpy(&b, &nd.state, 1);
        innernode[i] = b;
        mass[i] = nd.mass;
        xcom[i] = nd.xcom;
        ycom[i] = nd.ycom;
        r[i] = nd.r;
    }
    std::memcpy(expansions, Tree::expansions, sizeof(double) * 2 * ORDER * (size_t)n);
    std::memcpy(xs, Tree::xdata, sizeof(double) * (size_t)nsrc);
    std::memcpy(ys, Tree::ydata, sizeof(double) * (size_t)nsrc);
    std::memcpy(vs, Tree::vdata, sizeof(double) * (size_t)nsrc);
    bbox3[0] = Tree::xmin;
    bbox3[1] = Tree::ymin;
    bbox3[2] = Tree::ext;

    Tree::dispose();
    return n;
}
