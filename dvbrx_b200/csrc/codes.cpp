#include "codes.h"

#include <string.h>

#include <algorithm>

#include "codes_gen.h"

namespace drxg {

int find_table(int short_frame, const char* rate)
{
    if (!rate)
        return -1;
    const cg_rate* map = short_frame ? cg_rates_short : cg_rates_normal;
    const int n = short_frame ? (int)(sizeof(cg_rates_short) / sizeof(*cg_rates_short))
                              : (int)(sizeof(cg_rates_normal) / sizeof(*cg_rates_normal));
    for (int i = 0; i < n; i++)
        if (!strcmp(map[i].rate, rate))
            return map[i].table;
    return -1;
}

int degree_class(int deg_max)
{
    for (int k = 0; k < kNumClasses; k++)
        if (deg_max <= kClassDeg[k])
            return k;
    return -1;
}

bool compile_code(int table, Code* c, std::string* err)
{
    if (table < 0 || table >= CG_NTABLES) {
        *err = "no such table";
        return false;
    }
    const cg_table& t = cg_tables[table];
    c->table = table;
    c->table_name = t.name;
    c->N = t.N;
    c->K = t.K;
    c->R = t.N - t.K;
    c->q = c->R / QC;
    if (c->R % QC || c->K % QC || c->q < 1 || c->q > 255) {
        *err = "table is not quasi-cyclic with 360 columns";
        return false;
    }
    const int q = c->q;

    /* per layer: (g, a) pairs, in table order */
    std::vector<std::vector<std::pair<int, int>>> layer(q);
    c->addr.clear();
    c->aoff.assign(1, 0);
    const uint16_t* a = t.addr;
    int g = 0;
    for (int r = 0; r < t.nruns; r++) {
        const int deg = t.runs[2 * r];
        for (int k = 0; k < t.runs[2 * r + 1]; k++, g++, a += deg) {
            for (int n = 0; n < deg; n++) {
                if (a[n] >= c->R) {
                    *err = "accumulator address out of range";
                    return false;
                }
                layer[a[n] % q].push_back({g, a[n] / q});
                c->addr.push_back(a[n]);
            }
            c->aoff.push_back((uint32_t)c->addr.size());
        }
    }
    if (g * QC != c->K) {
        *err = "group count does not match K";
        return false;
    }
    /* Within a layer, the entries whose column group occurs more than once
     * (the only links two checks of the layer can share) go first, in table
     * order, then the rest.  A check node's result does not depend on the
     * order of its links (minimums and sign parity are symmetric, each link's
     * update is its own, and equal minimums give equal messages whichever
     * link holds the index), so this changes no output; it puts the links the
     * wavefront levels carry in the first slots. */
    for (int i = 0; i < q; i++) {
        auto shared = [&](const std::pair<int, int>& e) {
            int n = 0;
            for (auto& f : layer[i])
                n += f.first == e.first;
            return n > 1;
        };
        std::stable_partition(layer[i].begin(), layer[i].end(), shared);
    }

    c->ent.clear();
    c->eoff.assign(1, 0);
    c->cnt_max = 0;
    c->cnt_min = 1 << 30;
    int info_links = 0;
    for (int i = 0; i < q; i++) {
        for (auto& e : layer[i]) {
            c->ent.push_back(QC * e.first - e.second);
            c->ent.push_back(e.second);
        }
        c->eoff.push_back((uint16_t)(c->ent.size() / 2));
        c->cnt_max = std::max<int>(c->cnt_max, (int)layer[i].size());
        c->cnt_min = std::min<int>(c->cnt_min, (int)layer[i].size());
        info_links += (int)layer[i].size() * QC;
    }
    c->deg_max = c->cnt_max + 2;
    c->dclass = degree_class(c->deg_max);
    if (c->deg_max > 32) {
        *err = "check degree above 32";
        return false;
    }
    c->edges = info_links + 2 * c->R - 1;

    /* duplicate links inside one check would make the reference's in-order
     * writes observable: refuse such a table */
    for (int i = 0; i < q; i++)
        for (size_t x = 0; x < layer[i].size(); x++)
            for (size_t y = x + 1; y < layer[i].size(); y++)
                if (layer[i][x] == layer[i][y]) {
                    *err = "duplicate link in a check node";
                    return false;
                }

    /* levels inside each layer */
    c->steps.clear();
    c->perm.assign((size_t)q * QC, 0);
    c->nlev.assign(q, 1);
    c->lmeta.assign((size_t)q * QC, 0);
    c->levelled = false;
    c->phased = true;
    c->nlevels = 0;
    for (int i = 0; i < q; i++) {
        /* per check j: which of its information slots share their bit with
         * an earlier (in) or a later (out) check of the layer */
        const int ne = (int)layer[i].size();
        for (int j = 0; j < QC; j++) {
            uint64_t in = 0, out = 0;
            for (int x = 0; x < ne; x++)
                for (int y = 0; y < ne; y++) {
                    if (x == y || layer[i][x].first != layer[i][y].first)
                        continue;
                    /* bit of slot x of check j is slot y's bit of check jp */
                    const int jp = ((j - layer[i][x].second + layer[i][y].second) % QC + QC) % QC;
                    if (jp < j)
                        in |= 1ull << (2 + x);
                    else if (jp > j)
                        out |= 1ull << (2 + x);
                }
            /* masks of 24 slots: the shared links come first, so only a
             * layer with more than 22 of them would need more (it keeps
             * none, and the phased schedule does not run it) */
            if (((in | out) >> 24) == 0)
                c->lmeta[(size_t)i * QC + j] = in << 8 | out << 32;
            else
                c->phased = false;
        }
        std::vector<int> offs; /* d: check j shares a bit with check (j + d) mod 360 */
        for (size_t x = 0; x < layer[i].size(); x++)
            for (size_t y = 0; y < layer[i].size(); y++)
                if (x != y && layer[i][x].first == layer[i][y].first)
                    offs.push_back(((layer[i][y].second - layer[i][x].second) % QC + QC) % QC);
        std::vector<int> lev(QC, 0);
        int nl = 1;
        if (!offs.empty()) {
            for (int j = 0; j < QC; j++) {
                int l = 0;
                for (int d : offs) {
                    const int jp = (j + d) % QC;
                    if (jp < j)
                        l = std::max(l, lev[jp] + 1);
                }
                lev[j] = l;
                nl = std::max(nl, l + 1);
            }
        }
        const bool perm = nl > 1;
        c->levelled |= perm;
        c->nlev[i] = (uint8_t)nl;
        for (int j = 0; j < QC; j++)
            c->lmeta[(size_t)i * QC + j] |= (uint64_t)lev[j];
        int pos = 0;
        for (int l = 0; l < nl; l++) {
            const int start = pos;
            for (int j = 0; j < QC; j++)
                if (lev[j] == l)
                    c->perm[(size_t)i * QC + pos++] = (uint16_t)j;
            const int count = pos - start;
            c->steps.push_back((uint32_t)i | (uint32_t)start << 8 | (uint32_t)count << 17 |
                               (uint32_t)(perm ? 1 : 0) << 26);
        }
        c->nlevels += nl;
    }
    return true;
}

}  // namespace drxg
