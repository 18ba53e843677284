// Host-side mesh preprocessing for the membrane solid step (runs on the CPU).
//
//  * cvfes_mesh_incidence: node -> incident element slots, each node's elements
//    ordered as a fan (consecutive elements share an edge through the node), so
//    the gather kernel can carry one neighbour's displacement from one element
//    to the next.  The reference finds node/element neighbours with Python lists
//    (meshColoring.py:25-36); the row layout plays the role of the block-CSR row
//    of sparse.py:36-64 in the per-step Ku.
//  * cvfes_mesh_color_greedy: smallest-free-colour greedy colouring in element
//    order over the node-sharing graph, the algorithm of meshColoring.py:39-56.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "cvfes_b200.h"
#include "errors.h"

namespace {

struct Item {
    int32_t e, la, x, y;
};

}  // namespace

extern "C" int cvfes_mesh_incidence(int64_t n_nodes, int64_t n_elems, const int64_t* elems,
                                    int32_t* node_ptr, int32_t* slot_rec, int32_t* elem_slot) {
    if (n_nodes <= 0 || n_elems < 0 || (n_elems > 0 && !elems) || !node_ptr || !slot_rec ||
        !elem_slot)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_incidence: null pointer or bad size");
    if (n_nodes >= INT32_MAX || 3 * n_elems >= INT32_MAX)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_incidence: mesh too large for int32 slots");
    std::vector<int32_t> deg(n_nodes + 1, 0);
    for (int64_t e = 0; e < n_elems; ++e)
        for (int k = 0; k < 3; ++k) {
            int64_t a = elems[3 * e + k];
            if (a < 0 || a >= n_nodes)
                return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_incidence: node id out of range");
            deg[a + 1]++;
        }
    for (int64_t e = 0; e < n_elems; ++e)
        if (elems[3 * e] == elems[3 * e + 1] || elems[3 * e] == elems[3 * e + 2] ||
            elems[3 * e + 1] == elems[3 * e + 2])
            return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_incidence: degenerate element");
    node_ptr[0] = 0;
    for (int64_t a = 0; a < n_nodes; ++a) node_ptr[a + 1] = node_ptr[a] + deg[a + 1];

    // Gather the (element, local index) items per node, in element order.
    std::vector<int32_t> fill(n_nodes, 0);
    std::vector<Item> items(3 * n_elems);
    for (int64_t e = 0; e < n_elems; ++e)
        for (int la = 0; la < 3; ++la) {
            int64_t a = elems[3 * e + la];
            Item it;
            it.e = (int32_t)e;
            it.la = la;
            it.x = (int32_t)elems[3 * e + (la + 1) % 3];
            it.y = (int32_t)elems[3 * e + (la + 2) % 3];
            items[node_ptr[a] + fill[a]++] = it;
        }

    // Order each node's items as fans: start where an x is nobody's y (open fan)
    // else at the lowest element id; follow y -> x; restart on breaks.
    std::vector<Item> row, out;
    std::vector<char> used;
    for (int64_t a = 0; a < n_nodes; ++a) {
        const int32_t b = node_ptr[a], n = node_ptr[a + 1] - b;
        row.assign(items.begin() + b, items.begin() + b + n);
        used.assign(n, 0);
        out.clear();
        while ((int32_t)out.size() < n) {
            int start = -1;
            for (int i = 0; i < n && start < 0; ++i) {
                if (used[i]) continue;
                bool is_tail = false;
                for (int j = 0; j < n; ++j)
                    if (!used[j] && j != i && row[j].y == row[i].x) { is_tail = true; break; }
                if (!is_tail) start = i;
            }
            if (start < 0)
                for (int i = 0; i < n; ++i)
                    if (!used[i] && (start < 0 || row[i].e < row[start].e)) start = i;
            int cur = start;
            while (cur >= 0) {
                used[cur] = 1;
                out.push_back(row[cur]);
                int nxt = -1;
                for (int j = 0; j < n; ++j)
                    if (!used[j] && row[j].x == row[cur].y && (nxt < 0 || row[j].e < row[nxt].e))
                        nxt = j;
                cur = nxt;
            }
        }
        for (int i = 0; i < n; ++i) {
            const Item& it = out[i];
            const int32_t s = b + i;
            const bool cont = i > 0 && out[i - 1].y == it.x;
            slot_rec[4 * s + 0] = it.e;
            slot_rec[4 * s + 1] = it.x;
            slot_rec[4 * s + 2] = it.y;
            slot_rec[4 * s + 3] = (cont ? 1 : 0) | (it.la << 8);
            elem_slot[3 * (int64_t)it.e + it.la] = s;
        }
    }
    return CVFES_OK;
}

extern "C" int cvfes_mesh_color_greedy(int64_t n_nodes, int64_t n_elems, const int64_t* elems,
                                       int32_t max_colors, int32_t* colors) {
    if (n_nodes <= 0 || n_elems < 0 || !elems || !colors || max_colors <= 0)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_color_greedy: bad argument");
    std::vector<int64_t> ptr(n_nodes + 1, 0);
    for (int64_t i = 0; i < 3 * n_elems; ++i) {
        if (elems[i] < 0 || elems[i] >= n_nodes)
            return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_color_greedy: node id out of range");
        ptr[elems[i] + 1]++;
    }
    for (int64_t a = 0; a < n_nodes; ++a) ptr[a + 1] += ptr[a];
    std::vector<int64_t> adj(ptr[n_nodes]), fill(n_nodes, 0);
    for (int64_t e = 0; e < n_elems; ++e)
        for (int k = 0; k < 3; ++k) {
            int64_t a = elems[3 * e + k];
            adj[ptr[a] + fill[a]++] = e;
        }
    std::vector<int64_t> stamp(max_colors + 1, -1);
    int32_t used_colors = 0;
    for (int64_t e = 0; e < n_elems; ++e) colors[e] = -1;
    for (int64_t e = 0; e < n_elems; ++e) {
        for (int k = 0; k < 3; ++k) {
            int64_t a = elems[3 * e + k];
            for (int64_t q = ptr[a]; q < ptr[a + 1]; ++q) {
                int32_t c = colors[adj[q]];
                if (c >= 0) stamp[c] = e;
            }
        }
        int32_t c = 0;
        while (c < max_colors && stamp[c] == e) ++c;
        if (c == max_colors)
            return cvfes::fail(CVFES_ERR_MESH, "cvfes_mesh_color_greedy: colours are used up");
        colors[e] = c;
        used_colors = std::max(used_colors, c + 1);
    }
    return used_colors;
}
