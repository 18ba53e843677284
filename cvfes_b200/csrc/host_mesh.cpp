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

namespace {

// Cover the sorted distinct ids with at most `max_w` windows of `h` consecutive ids,
// greedily from the smallest uncovered id (the fewest windows for fixed-length
// intervals); returns the window starts.
std::vector<int32_t> cover_windows(const std::vector<int32_t>& ids, int32_t h, int32_t max_w) {
    std::vector<int32_t> starts;
    size_t i = 0;
    while (i < ids.size() && (int32_t)starts.size() < max_w) {
        const int32_t s = ids[i];
        starts.push_back(s);
        while (i < ids.size() && ids[i] < s + h) ++i;
    }
    return starts;
}

// Shared-memory row of id within the windows (window k holds ids [starts[k], +h)),
// or -1 - id when no window holds it.
int32_t window_loc(const std::vector<int32_t>& starts, int32_t h, int32_t id) {
    for (size_t k = 0; k < starts.size(); ++k)
        if (id >= starts[k] && id < starts[k] + h) return (int32_t)k * h + (id - starts[k]);
    return -1 - id;
}

}  // namespace

extern "C" int cvfes_mesh_tiles(int64_t n_nodes, int64_t n_elems, const int32_t* node_ptr,
                                const int32_t* slot_rec, int64_t n_clamped, int32_t P, int32_t H,
                                int32_t W, int32_t EH, int32_t WE, int32_t* tile_win,
                                int32_t* tile_rec, int32_t* node_loc, int64_t* stats) {
    if (n_nodes <= 0 || n_elems <= 0 || !node_ptr || !slot_rec || !tile_win || !tile_rec ||
        !node_loc || !stats || P < 1 || H < P || W < 1 || EH < 1 || WE < 1 || n_clamped < 0 ||
        n_clamped > n_nodes)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_mesh_tiles: bad argument");
    const int64_t n_tiles = (n_nodes + P - 1) / P;
    const int nw = W + WE;
    int64_t out_nodes = 0, out_elems = 0, max_need = 0;
    std::vector<int32_t> nid, eid;
    for (int64_t t = 0; t < n_tiles; ++t) {
        const int64_t a0 = t * P, a1 = std::min<int64_t>(a0 + P, n_nodes);
        nid.clear();
        eid.clear();
        for (int64_t a = std::max<int64_t>(a0, n_clamped); a < a1; ++a) {
            nid.push_back((int32_t)a);
            for (int32_t k = node_ptr[a]; k < node_ptr[a + 1]; ++k) {
                eid.push_back(slot_rec[4 * (int64_t)k]);
                nid.push_back(slot_rec[4 * (int64_t)k + 1]);
                nid.push_back(slot_rec[4 * (int64_t)k + 2]);
            }
        }
        std::sort(nid.begin(), nid.end());
        nid.erase(std::unique(nid.begin(), nid.end()), nid.end());
        std::sort(eid.begin(), eid.end());
        eid.erase(std::unique(eid.begin(), eid.end()), eid.end());
        const std::vector<int32_t> ns = cover_windows(nid, H, W);
        const std::vector<int32_t> es = cover_windows(eid, EH, WE);
        const int64_t need = (int64_t)cover_windows(nid, H, 1 << 20).size();
        max_need = std::max(max_need, need);
        for (int k = 0; k < nw; ++k) tile_win[t * nw + k] = -1;
        for (size_t k = 0; k < ns.size(); ++k) tile_win[t * nw + k] = ns[k];
        for (size_t k = 0; k < es.size(); ++k) tile_win[t * nw + W + k] = es[k];
        for (int64_t a = a0; a < a1; ++a) {
            const bool live = a >= n_clamped;
            node_loc[a] = live ? window_loc(ns, H, (int32_t)a) : -1 - (int32_t)a;
            for (int32_t k = node_ptr[a]; k < node_ptr[a + 1]; ++k) {
                const int64_t q = 4 * (int64_t)k;
                const int32_t e = slot_rec[q], b1 = slot_rec[q + 1], b2 = slot_rec[q + 2];
                tile_rec[q] = live ? window_loc(es, EH, e) : -1 - e;
                tile_rec[q + 1] = live ? window_loc(ns, H, b1) : -1 - b1;
                tile_rec[q + 2] = live ? window_loc(ns, H, b2) : -1 - b2;
                tile_rec[q + 3] = slot_rec[q + 3];
                if (live) {
                    out_elems += tile_rec[q] < 0;
                    out_nodes += (tile_rec[q + 1] < 0) + (tile_rec[q + 2] < 0);
                }
            }
        }
    }
    stats[0] = n_tiles;
    stats[1] = out_nodes;
    stats[2] = out_elems;
    stats[3] = max_need;
    return CVFES_OK;
}
