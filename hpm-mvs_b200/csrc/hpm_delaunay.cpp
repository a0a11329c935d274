/*
 * Incremental Delaunay triangulation (Bowyer-Watson) of the support points,
 * replacing cv::Subdiv2D in DelaunayTriangulation (HPM.cpp:787-809).
 *
 * Exact integer predicates: coordinates are pixel positions (< 16384), the
 * enclosing triangle's corners stay below 2^17, so every orientation
 * determinant fits in 64-bit integers and every in-circle determinant in
 * 128-bit ones.  Points are located by a
 * visibility walk from the last created triangle; support points arrive in
 * the reference's block order (column-major 5x5 blocks), so consecutive
 * points are neighbours and the walk is short.
 */
#include <cstdint>
#include <vector>

#include "hpm_prior.h"

namespace hpm {
namespace {

struct Tri {
    int v[3];  /* counter-clockwise */
    int nb[3]; /* neighbour across the edge opposite v[i], -1 = none */
    bool alive;
};

struct Pt {
    int64_t x, y;
};

inline int64_t orient(const Pt &a, const Pt &b, const Pt &c)
{
    return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
}

/* > 0 when d lies strictly inside the circumcircle of the ccw triangle abc */
inline bool in_circle(const Pt &a, const Pt &b, const Pt &c, const Pt &d)
{
    const int64_t adx = a.x - d.x, ady = a.y - d.y, bdx = b.x - d.x, bdy = b.y - d.y, cdx = c.x - d.x, cdy = c.y - d.y;
    const int64_t al = adx * adx + ady * ady, bl = bdx * bdx + bdy * bdy, cl = cdx * cdx + cdy * cdy;
    const __int128 det = (__int128)adx * (bdy * cl - bl * cdy) - (__int128)ady * (bdx * cl - bl * cdx) +
                         (__int128)al * (bdx * cdy - bdy * cdx);
    return det > 0;
}

}  // namespace

void delaunay(const std::vector<int> &xy, int w, int h, std::vector<int> &out)
{
    out.clear();
    const int n = (int)xy.size() / 2;
    if (n < 3) return;
    std::vector<Pt> P(n + 3);
    for (int i = 0; i < n; ++i) P[i] = {xy[2 * i], xy[2 * i + 1]};
    /* the enclosing triangle of cv::Subdiv2D::initDelaunay (OpenCV 4.x) for
     * the rect (0, 0, w, h): corners (6M, 0), (0, 6M), (-6M, -6M),
     * M = max(w, h).  The triangles along the hull depend on it: a sliver
     * on the hull survives only while no corner lies in its circumcircle. */
    const int64_t M3 = 6 * (int64_t)(w > h ? w : h);
    P[n] = {M3, 0};
    P[n + 1] = {0, M3};
    P[n + 2] = {-M3, -M3};
    std::vector<Tri> T;
    T.reserve(2 * n + 8);
    T.push_back({{n, n + 1, n + 2}, {-1, -1, -1}, true});
    int last = 0;
    std::vector<int> cavity, stack, mark(1, 0);
    int stamp = 0;
    struct BEdge {
        int a, b, outer;
    };
    std::vector<BEdge> boundary;
    for (int ip = 0; ip < n; ++ip) {
        const Pt &p = P[ip];
        /* visibility walk to a triangle containing p */
        int t = last;
        if (!T[t].alive) {
            for (t = (int)T.size() - 1; t >= 0 && !T[t].alive; --t) {
            }
        }
        for (int guard = 0; guard < 4 * (int)T.size() + 16; ++guard) {
            const Tri &tr = T[t];
            int next = -1;
            for (int e = 0; e < 3; ++e) {
                if (orient(P[tr.v[(e + 1) % 3]], P[tr.v[(e + 2) % 3]], p) < 0) {
                    next = tr.nb[e];
                    break;
                }
            }
            if (next < 0) break;
            t = next;
        }
        /* cavity: triangles whose circumcircle strictly contains p */
        ++stamp;
        if (mark.size() < T.size()) mark.resize(T.size(), 0);
        cavity.clear();
        stack.clear();
        stack.push_back(t);
        mark[t] = stamp;
        while (!stack.empty()) {
            const int c = stack.back();
            stack.pop_back();
            cavity.push_back(c);
            for (int e = 0; e < 3; ++e) {
                const int o = T[c].nb[e];
                if (o < 0 || mark[o] == stamp) continue;
                const Tri &to = T[o];
                if (in_circle(P[to.v[0]], P[to.v[1]], P[to.v[2]], p)) {
                    mark[o] = stamp;
                    stack.push_back(o);
                }
            }
        }
        /* boundary edges of the cavity, ccw as seen from inside */
        boundary.clear();
        for (int c : cavity) {
            for (int e = 0; e < 3; ++e) {
                const int o = T[c].nb[e];
                if (o >= 0 && mark[o] == stamp) continue;
                boundary.push_back({T[c].v[(e + 1) % 3], T[c].v[(e + 2) % 3], o});
            }
            T[c].alive = false;
        }
        /* fan of new triangles (p, a, b); link them through their shared
         * edges (p, a) / (b, p) */
        const int first = (int)T.size();
        for (const BEdge &be : boundary) {
            Tri nt;
            nt.v[0] = ip;
            nt.v[1] = be.a;
            nt.v[2] = be.b;
            nt.nb[0] = be.outer; /* edge (a, b) opposite p */
            nt.nb[1] = -1;
            nt.nb[2] = -1;
            nt.alive = true;
            const int id = (int)T.size();
            T.push_back(nt);
            if (be.outer >= 0) {
                Tri &o = T[be.outer];
                for (int e = 0; e < 3; ++e)
                    if (o.v[(e + 1) % 3] == be.b && o.v[(e + 2) % 3] == be.a) o.nb[e] = id;
            }
        }
        const int cnt = (int)T.size() - first;
        /* edge (b, p) of triangle i (opposite v[1]=a) meets edge (p, a') of
         * the triangle whose a' == b (opposite v[2]) */
        for (int i = 0; i < cnt; ++i) {
            Tri &ti = T[first + i];
            for (int j = 0; j < cnt; ++j) {
                if (i == j) continue;
                if (T[first + j].v[1] == ti.v[2]) {
                    ti.nb[1] = first + j;
                    T[first + j].nb[2] = first + i;
                    break;
                }
            }
        }
        last = (int)T.size() - 1;
        if (mark.size() < T.size()) mark.resize(T.size(), 0);
    }
    for (const Tri &t : T) {
        if (!t.alive || t.v[0] >= n || t.v[1] >= n || t.v[2] >= n) continue;
        bool inside = true;
        for (int k = 0; k < 3; ++k) {
            const Pt &q = P[t.v[k]];
            if (!(q.x >= 0 && q.x < w && q.y >= 0 && q.y < h)) inside = false;
        }
        if (!inside) continue;
        for (int k = 0; k < 3; ++k) {
            out.push_back((int)P[t.v[k]].x);
            out.push_back((int)P[t.v[k]].y);
        }
    }
}

}  // namespace hpm

extern "C" int hpm_delaunay(const int *xy, int n, int w, int h, int *tris_out, int cap)
{
    if ((!xy && n > 0) || n < 0 || w < 1 || h < 1) return HPM_ERR_ARG;
    std::vector<int> pts(xy, xy + 2 * n), tris;
    hpm::delaunay(pts, w, h, tris);
    const int nt = (int)tris.size() / 6;
    if (tris_out) {
        if (nt > cap) return HPM_ERR_ARG;
        for (size_t i = 0; i < tris.size(); ++i) tris_out[i] = tris[i];
    }
    return nt;
}
