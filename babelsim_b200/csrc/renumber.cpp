// Locality renumbering of the cells of a mesh (host, once per mesh).
//
// The persistent sweeps read each row's neighbours' values through the SELL-32
// slices of 32 consecutive rows, so they coalesce when neighbouring cells have
// nearby numbers.  A mesh read from a file can be numbered arbitrarily; then the
// cells are renumbered by reverse Cuthill-McKee on the cell graph (one
// breadth-first ordering per connected component, started from a
// pseudo-peripheral cell, neighbours taken by increasing degree, the
// component's order reversed), components kept in the order of their lowest
// cell number, so independent cases concatenated into one mesh keep their cell
// ranges.  A mesh that is already local (mean |i - j| over interior faces within
// twice the reverse Cuthill-McKee order's) keeps its numbering: the generated
// lattice-ordered meshes coalesce best as they are.
#include "renumber.h"

#include <algorithm>
#include <cstdlib>

namespace bsg {
namespace {

// breadth-first levels from `start` within the unvisited cells; returns the visit order
std::vector<int> bfs(int start, const std::vector<int>& ptr, const std::vector<int>& adj, std::vector<int>& mark,
                     int stamp, bool by_degree) {
    std::vector<int> order{start};
    mark[start] = stamp;
    std::vector<int> nb;
    for (std::size_t head = 0; head < order.size(); ++head) {
        const int c = order[head];
        nb.clear();
        for (int k = ptr[c]; k < ptr[c + 1]; ++k)
            if (mark[adj[k]] != stamp) {
                mark[adj[k]] = stamp;
                nb.push_back(adj[k]);
            }
        if (by_degree)
            std::stable_sort(nb.begin(), nb.end(),
                             [&](int a, int b) { return ptr[a + 1] - ptr[a] < ptr[b + 1] - ptr[b]; });
        order.insert(order.end(), nb.begin(), nb.end());
    }
    return order;
}

double meanSpan(int F, const int* owner, const int* nbr, const std::vector<int>& pos) {
    double s = 0.0;
    long long n = 0;
    for (int f = 0; f < F; ++f) {
        if (nbr[f] < 0) continue;
        s += std::abs(pos[owner[f]] - pos[nbr[f]]);
        ++n;
    }
    return n ? s / static_cast<double>(n) : 0.0;
}

}  // namespace

std::vector<int> localityOrder(int N, int F, const int* owner, const int* nbr, bool* applied) {
    std::vector<int> ptr(N + 1, 0);
    for (int f = 0; f < F; ++f)
        if (nbr[f] >= 0) {
            ++ptr[owner[f] + 1];
            ++ptr[nbr[f] + 1];
        }
    for (int c = 0; c < N; ++c) ptr[c + 1] += ptr[c];
    std::vector<int> adj(ptr[N]);
    {
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int f = 0; f < F; ++f)
            if (nbr[f] >= 0) {
                adj[fill[owner[f]]++] = nbr[f];
                adj[fill[nbr[f]]++] = owner[f];
            }
    }
    std::vector<int> order;
    order.reserve(N);
    std::vector<int> mark(N, -1), done(N, 0);
    int stamp = 0;
    for (int first = 0; first < N; ++first) {
        if (done[first]) continue;
        // pseudo-peripheral start: the last cell reached from the component's lowest-numbered cell
        const std::vector<int> probe = bfs(first, ptr, adj, mark, stamp++, false);
        const std::vector<int> comp = bfs(probe.back(), ptr, adj, mark, stamp++, true);
        for (auto it = comp.rbegin(); it != comp.rend(); ++it) {
            order.push_back(*it);
            done[*it] = 1;
        }
    }
    std::vector<int> pos(N), ident(N);
    for (int i = 0; i < N; ++i) {
        pos[order[i]] = i;
        ident[i] = i;
    }
    const bool apply = meanSpan(F, owner, nbr, ident) > 2.0 * meanSpan(F, owner, nbr, pos);
    if (applied) *applied = apply;
    if (!apply) return ident;
    return order;
}

}  // namespace bsg
