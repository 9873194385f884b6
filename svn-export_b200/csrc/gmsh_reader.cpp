// gmsh 2.2 ASCII input: meshes (GmshMeshReader::read_mesh, src/mesh/msh_gmshreader.cc:75-244,
// with the region rules of RegionDB::add_region, src/mesh/region.cc:107-175) and element
// fields (read_data_header / read_element_data, msh_gmshreader.cc:251-396).
//
// The reference reads token by token through a line tokenizer.  Here the file is read into
// memory once and its content lines -- the lines Tokenizer::next_line stops at
// (src/system/tokenizer.cc:72-100): not blank, not starting with '#' after trimming -- are
// indexed by all threads, each over its own byte range.  The node, element and data rows,
// whose positions are then known, are parsed in parallel straight into their final slots;
// the bookkeeping whose outcome depends on file order (regions created on first appearance,
// repeated ids, which error comes first) runs as one ordered pass over the parsed rows.
// Every error names the first offending line of the file, as the reference's sequential
// reading would.
#include <fcntl.h>
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "mesh_store.hpp"
#include "mh_darcy.h"

namespace {

constexpr int64_t kNone = std::numeric_limits<int64_t>::max();

struct Text {
    std::unique_ptr<char[]> data;
    int64_t size = 0;
    std::string path;
    std::unique_ptr<int64_t[]> line;  // offset of the first non-blank character of each content line
    int64_t n_line = 0;

    const char *end() const { return data.get() + size; }
    // 1-based line number of the file for byte offset `off` (error messages only)
    int64_t file_line(int64_t off) const {
        int64_t n = 1;
        const char *p = data.get(), *e = p + off;
        while ((p = static_cast<const char *>(std::memchr(p, '\n', e - p)))) ++n, ++p;
        return n;
    }
    std::string where(int64_t k) const {
        if (k >= n_line) return path + ": end of file";
        return path + ":" + std::to_string(file_line(line[k]));
    }
};

inline bool trim_char(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// Reads the whole file: fstat for the size, then every thread preads its share of the bytes
// (a regular file in the page cache is copied at memory speed by all cores at once).
int load(const char *path, Text &t, std::string &err) {
    t.path = path;
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) {
        err = std::string("cannot open '") + path + "'";
        return MH_ERR_IO;
    }
    struct stat st;
    int rc = (::fstat(fd, &st) != 0 || !S_ISREG(st.st_mode)) ? MH_ERR_IO : MH_OK;
    const int64_t sz = rc ? 0 : (int64_t)st.st_size;
    if (!rc) {
        t.data.reset(new (std::nothrow) char[sz > 0 ? sz : 1]);
        if (!t.data) rc = MH_ERR_NOMEM;
    }
    if (!rc && sz > 0) {
        const int nt = sz < (8 << 20) ? 1 : omp_get_max_threads();
        int bad = 0;
#pragma omp parallel num_threads(nt) reduction(| : bad)
        {
            const int k = omp_get_thread_num();
            int64_t lo = sz * k / nt;
            const int64_t hi = sz * (k + 1) / nt;
            while (lo < hi) {
                const ssize_t r = ::pread(fd, t.data.get() + lo, (size_t)(hi - lo), (off_t)lo);
                if (r <= 0) {
                    bad = 1;
                    break;
                }
                lo += r;
            }
        }
        if (bad) rc = MH_ERR_IO;
    }
    t.size = sz;
    ::close(fd);
    if (rc == MH_ERR_IO) err = std::string("cannot read '") + path + "'";
    if (rc == MH_ERR_NOMEM) err = "out of host memory reading '" + std::string(path) + "'";
    if (rc) return rc;

    // Index the content lines.  Thread k owns the lines that start in its byte range.
    const char *b = t.data.get();
    const int64_t n = t.size;
    const int nt = n < (1 << 20) ? 1 : omp_get_max_threads();
    std::vector<std::vector<int64_t>> part(nt);
    std::vector<int64_t> start(nt + 1, 0);
#pragma omp parallel num_threads(nt)
    {
        const int k = omp_get_thread_num();
        const int64_t lo = n * k / nt, hi = n * (k + 1) / nt;
        int64_t p = lo;
        if (p > 0) {  // first line start >= lo: lines start at 0 and after each '\n'
            const void *q = std::memchr(b + p - 1, '\n', n - (p - 1));
            p = q ? static_cast<const char *>(q) - b + 1 : n;
        }
        std::vector<int64_t> &out = part[k];
        out.reserve((hi - lo) / 24 + 16);
        while (p < hi) {
            const void *q = std::memchr(b + p, '\n', n - p);
            const int64_t e = q ? static_cast<const char *>(q) - b : n;
            int64_t s = p;
            while (s < e && trim_char(b[s])) ++s;
            if (s < e && b[s] != '#') out.push_back(s);
            p = e + 1;
        }
        start[k + 1] = (int64_t)out.size();
#pragma omp barrier
#pragma omp single
        {
            for (int q = 0; q < nt; ++q) start[q + 1] += start[q];
            t.n_line = start[nt];
            t.line.reset(new int64_t[t.n_line > 0 ? t.n_line : 1]);
        }
        std::copy(out.begin(), out.end(), t.line.get() + start[k]);
    }
    return MH_OK;
}

// Tokens of one content line: separated by blanks, '"' quoting (separators inside quotes
// are part of the token, the quotes are dropped) and '\' escaping the next character, as
// boost::escaped_list_separator("\\", " \t", "\"") with empty tokens dropped.
struct Line {
    const char *p, *e;
    std::string scratch;

    Line(const Text &t, int64_t k) {
        p = t.data.get() + t.line[k];
        const void *q = std::memchr(p, '\n', t.end() - p);
        e = q ? static_cast<const char *>(q) : t.end();
        while (e > p && trim_char(e[-1])) --e;
    }
    // next token as [b, x); quoted or escaped tokens are unescaped into `scratch`
    bool next(const char *&b, const char *&x) {
        while (p < e && (*p == ' ' || *p == '\t')) ++p;
        if (p >= e) return false;
        const char *s = p;
        bool plain = true;
        while (p < e && *p != ' ' && *p != '\t') {
            if (*p == '"' || *p == '\\') {
                plain = false;
                break;
            }
            ++p;
        }
        if (plain) {
            b = s;
            x = p;
            return true;
        }
        scratch.assign(s, p);
        bool quoted = false;
        while (p < e) {
            char c = *p;
            if (c == '\\' && p + 1 < e) {
                c = *++p;
                if (c == 'n') c = '\n';
                scratch.push_back(c);
            } else if (c == '"') {
                quoted = !quoted;
            } else if (!quoted && (c == ' ' || c == '\t')) {
                break;
            } else {
                scratch.push_back(c);
            }
            ++p;
        }
        if (scratch.empty()) return next(b, x);  // "" is an empty token: dropped
        b = scratch.data();
        x = b + scratch.size();
        return true;
    }
    bool u32(uint32_t &v) {
        const char *b, *x;
        if (!next(b, x)) return false;
        if (b < x && *b == '+') ++b;
        if (b == x) return false;
        auto r = std::from_chars(b, x, v);
        return r.ec == std::errc() && r.ptr == x;
    }
    bool f64(double &v) {
        const char *b, *x;
        if (!next(b, x)) return false;
        if (b < x && *b == '+') ++b;
        if (b == x) return false;
        auto r = std::from_chars(b, x, v);
        return r.ec == std::errc() && r.ptr == x;
    }
    std::string str() {
        const char *b, *x;
        return next(b, x) ? std::string(b, x) : std::string();
    }
};

// First content line at or after k that contains `pat` (Tokenizer::skip_to); stops with
// kNone at the end of the file or at a line containing `stop`.
int64_t skip_to(const Text &t, int64_t k, const char *pat, const char *stop = nullptr) {
    const size_t lp = std::strlen(pat), ls = stop ? std::strlen(stop) : 0;
    for (; k < t.n_line; ++k) {
        Line l(t, k);
        std::string_view v(l.p, l.e - l.p);
        if (v.find(std::string_view(pat, lp)) != std::string_view::npos) return k;
        if (stop && v.find(std::string_view(stop, ls)) != std::string_view::npos) return kNone;
    }
    return kNone;
}

// The first error of an ordered set of rows: the smallest row wins.
struct FirstError {
    int64_t row = kNone;
    int stage = 0;
    std::string msg;
    void offer(int64_t r, int s, std::string m) {
        if (r < row || (r == row && s < stage)) {
            row = r;
            stage = s;
            msg = std::move(m);
        }
    }
};

struct Region {
    int32_t id, dim;
    bool boundary;
    std::string name;
};

struct RegionTable {
    std::vector<Region> list;
    std::unordered_map<int64_t, int32_t> by_id;
    std::unordered_map<std::string, int32_t> by_name;

    // RegionDB::add_region(id, label, dim, boundary), region.cc:107-149; "" on success
    std::string add_named(int64_t id, const std::string &name, int dim) {
        const bool bdr = !name.empty() && name[0] == '.';
        auto it = by_id.find(id);
        if (it != by_id.end()) {
            const Region &r = list[it->second];
            if (r.name != name)
                return "region id " + std::to_string(id) + " named '" + name + "' already names '" + r.name + "'";
            if (r.dim != dim)
                return "region '" + name + "' (id " + std::to_string(id) + ") given dimensions " +
                       std::to_string(r.dim) + " and " + std::to_string(dim);
            if (r.boundary != bdr) return "region '" + name + "' is both boundary and bulk";
            return "";
        }
        if (by_name.count(name))
            return "region name '" + name + "' of id " + std::to_string(id) + " already belongs to id " +
                   std::to_string(list[by_name[name]].id);
        if (id > std::numeric_limits<int32_t>::max()) return "region id " + std::to_string(id) + " out of range";
        by_id[id] = (int32_t)list.size();
        by_name[name] = (int32_t)list.size();
        list.push_back({(int32_t)id, dim, bdr, name});
        return "";
    }
    // RegionDB::add_region(id, dim), region.cc:164-175: the region of an element
    int32_t of_element(int64_t id, int dim, std::string &err) {
        auto it = by_id.find(id);
        if (it != by_id.end()) {
            const Region &r = list[it->second];
            if (r.dim != dim) {
                err = "element of dimension " + std::to_string(dim) + " in region '" + r.name + "' (id " +
                      std::to_string(id) + ") of dimension " + std::to_string(r.dim);
                return -1;
            }
            return it->second;
        }
        err = add_named(id, "region_" + std::to_string(id), dim);
        if (!err.empty()) return -1;
        list.back().boundary = false;
        return (int32_t)list.size() - 1;
    }
};

// Node id -> index: a dense table for ids up to a few times the node count, else a sorted
// list searched by bisection.
struct NodeIndex {
    std::vector<int32_t> dense;
    std::vector<std::pair<uint32_t, int32_t>> sorted;
    bool is_dense = true;

    int32_t find(uint32_t id) const {
        if (is_dense) return id < dense.size() ? dense[id] : -1;
        auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(id, INT32_MIN));
        return (it != sorted.end() && it->first == id) ? it->second : -1;
    }
    // builds the index of ids[n]; returns the row of the first repeated id, or kNone
    int64_t build(const std::vector<uint32_t> &ids, int64_t n) {
        uint32_t mx = 0;
#pragma omp parallel for reduction(max : mx) schedule(static)
        for (int64_t i = 0; i < n; ++i) mx = std::max(mx, ids[i]);
        is_dense = (uint64_t)mx <= 8 * (uint64_t)n + (1u << 20);
        if (is_dense) {
            dense.assign((size_t)mx + 1, -1);
            for (int64_t i = 0; i < n; ++i) {
                if (dense[ids[i]] >= 0) return i;
                dense[ids[i]] = (int32_t)i;
            }
            return kNone;
        }
        sorted.resize(n);
        for (int64_t i = 0; i < n; ++i) sorted[i] = {ids[i], (int32_t)i};
        std::sort(sorted.begin(), sorted.end());
        int64_t first = kNone;
        for (int64_t i = 1; i < n; ++i)
            if (sorted[i].first == sorted[i - 1].first && (i < 2 || sorted[i - 2].first != sorted[i].first))
                first = std::min<int64_t>(first, sorted[i].second);  // second occurrence of an id
        return first;
    }
};

// Repeated-id detection over ids met in order (ElementVector::add_item, sys_vector.hh:371).
struct IdSet {
    std::vector<uint8_t> seen;
    std::unordered_map<uint32_t, char> sparse;
    bool dense;
    explicit IdSet(uint32_t max_id, int64_t n) : dense((uint64_t)max_id <= 8 * (uint64_t)n + (1u << 20)) {
        if (dense) seen.assign((size_t)max_id + 1, 0);
    }
    bool insert(uint32_t id) {  // false if already present
        if (dense) {
            if (seen[id]) return false;
            seen[id] = 1;
            return true;
        }
        return sparse.emplace(id, 1).second;
    }
};

int read_mesh(const char *path, mh_mesh &out, std::string &err) {
    Text t;
    int rc = load(path, t, err);
    if (rc) return rc;
    const int64_t nl = t.n_line;
    auto fail = [&](int64_t k, const std::string &msg) {
        err = t.where(k) + ": " + msg;
        return MH_ERR_INVALID;
    };

    // $PhysicalNames (read_physical_names, msh_gmshreader.cc:220-244): searched before $Nodes
    RegionTable reg;
    int64_t cur = 0;
    int64_t k = skip_to(t, 0, "$PhysicalNames", "$Nodes");
    if (k != kNone) {
        if (k + 1 >= nl) return fail(k + 1, "missing count of $PhysicalNames");
        uint32_t n_ph;
        if (!Line(t, k + 1).u32(n_ph)) return fail(k + 1, "wrong format of number");
        for (uint32_t i = 0; i < n_ph; ++i) {
            const int64_t r = k + 2 + i;
            if (r >= nl) return fail(r, "unexpected end of file in $PhysicalNames");
            Line l(t, r);
            uint32_t dim, id;
            if (!l.u32(dim) || !l.u32(id)) return fail(r, "wrong format of number");
            std::string msg = reg.add_named(id, l.str(), (int)dim);
            if (!msg.empty()) return fail(r, msg);
        }
        cur = k + 1 + n_ph;
    }

    // $Nodes (read_nodes, msh_gmshreader.cc:89-117)
    k = skip_to(t, cur, "$Nodes");
    if (k == kNone) {
        err = t.path + ": missing section '$Nodes'";
        return MH_ERR_INVALID;
    }
    uint32_t nn32;
    if (k + 1 >= nl || !Line(t, k + 1).u32(nn32)) return fail(k + 1, "wrong format of number");
    const int64_t nn = nn32;
    if (nn == 0) return fail(k + 1, "zero number of nodes");
    if (nn > std::numeric_limits<int32_t>::max()) return fail(k + 1, "too many nodes");
    const int64_t n0 = k + 2;
    // rows present in the file (a count beyond the end of the file is an error at the end,
    // after the rows that are there, and allocates nothing for the missing ones)
    const int64_t n_avail = std::min<int64_t>(nn, std::max<int64_t>(0, nl - n0));
    std::vector<uint32_t> nid(n_avail);
    out.m.xyz.resize(n_avail * 3);
    FirstError node_err;
    {
        const int64_t avail = n_avail;
        if (avail < nn) node_err.offer(nl, 0, "unexpected end of file in $Nodes");
#pragma omp parallel
        {
            FirstError mine;
#pragma omp for schedule(static)
            for (int64_t i = 0; i < avail; ++i) {
                if (mine.row != kNone) continue;
                Line l(t, n0 + i);
                double *x = &out.m.xyz[3 * i];
                if (!l.u32(nid[i]) || !l.f64(x[0]) || !l.f64(x[1]) || !l.f64(x[2]))
                    mine.offer(n0 + i, 0, "wrong format of number");
            }
#pragma omp critical
            node_err.offer(mine.row, mine.stage, mine.msg);
        }
    }
    NodeIndex nodes;
    const int64_t ok_nodes = node_err.row == kNone ? nn : node_err.row - n0;
    const int64_t dup = nodes.build(nid, ok_nodes);
    if (dup != kNone) return fail(n0 + dup, "repeated node id " + std::to_string(nid[dup]));
    if (node_err.row != kNone) return fail(node_err.row, node_err.msg);

    // $Elements (read_elements, msh_gmshreader.cc:121-216)
    k = skip_to(t, n0 + nn - 1, "$Elements");
    if (k == kNone) {
        err = t.path + ": missing section '$Elements'";
        return MH_ERR_INVALID;
    }
    uint32_t ne32;
    if (k + 1 >= nl || !Line(t, k + 1).u32(ne32)) return fail(k + 1, "wrong format of number");
    const int64_t ne = ne32;
    if (ne == 0) return fail(k + 1, "zero number of elements");
    if (ne > std::numeric_limits<int32_t>::max()) return fail(k + 1, "too many elements");
    const int64_t e0 = k + 2;
    // per row present in the file (left uninitialised: every row the later passes read is written)
    const int64_t e_avail = std::min<int64_t>(ne, std::max<int64_t>(0, nl - e0));
    std::unique_ptr<uint32_t[]> eid(new uint32_t[e_avail + 1]), ereg(new uint32_t[e_avail + 1]);
    std::unique_ptr<int32_t[]> epart(new int32_t[e_avail + 1]), enodes(new int32_t[4 * e_avail + 4]);
    std::unique_ptr<int8_t[]> edim(new int8_t[e_avail + 1]), cls(new int8_t[e_avail + 1]);
    // stage 0: errors before the region is known; stage 1: errors in the node list, which
    // the reference meets after the region and id bookkeeping of the same line
    FirstError el_err;
    {
        const int64_t avail = e_avail;
        if (avail < ne) el_err.offer(nl, 0, "unexpected end of file in $Elements");
#pragma omp parallel
        {
            FirstError mine;
#pragma omp for schedule(static)
            for (int64_t i = 0; i < avail; ++i) {
                if (mine.row != kNone) continue;
                const int64_t r = e0 + i;
                Line l(t, r);
                uint32_t type, ntags, obj;
                std::fill(&enodes[4 * i], &enodes[4 * i] + 4, -1);
                if (!l.u32(eid[i]) || !l.u32(type)) {
                    mine.offer(r, 0, "wrong format of number");
                    continue;
                }
                int dim;
                switch (type) {
                    case 1: dim = 1; break;
                    case 2: dim = 2; break;
                    case 4: dim = 3; break;
                    case 15: dim = 0; break;
                    default:
                        mine.offer(r, 0, "element " + std::to_string(eid[i]) + " is of the unsupported type " +
                                             std::to_string(type));
                        continue;
                }
                edim[i] = (int8_t)dim;
                if (!l.u32(ntags)) {
                    mine.offer(r, 0, "wrong format of number");
                    continue;
                }
                if (ntags < 2) {
                    mine.offer(r, 0, "element " + std::to_string(eid[i]) + " has fewer than two tags");
                    continue;
                }
                uint32_t part = 0, skip;
                bool ok = l.u32(ereg[i]) && l.u32(obj) && (ntags < 3 || l.u32(part));
                for (uint32_t ti = 3; ok && ti < ntags; ++ti) ok = l.u32(skip);
                if (!ok) {
                    mine.offer(r, 0, "wrong format of number");
                    continue;
                }
                epart[i] = (int32_t)std::min<uint32_t>(part, (uint32_t)std::numeric_limits<int32_t>::max());
                for (int j = 0; j <= dim; ++j) {
                    uint32_t id;
                    if (!l.u32(id)) {
                        mine.offer(r, 1, "wrong format of number");
                        break;
                    }
                    const int32_t idx = nodes.find(id);
                    if (idx < 0) {
                        mine.offer(r, 1, "unknown node id " + std::to_string(id) + " in element " +
                                             std::to_string(eid[i]));
                        break;
                    }
                    enodes[4 * i + j] = idx;
                }
            }
#pragma omp critical
            el_err.offer(mine.row, mine.stage, mine.msg);
        }
    }

    // ordered pass: regions on first appearance, boundary or bulk, repeated element ids
    const int64_t last = el_err.row == kNone ? ne : el_err.row - e0 + (el_err.stage == 1 ? 1 : 0);
    {
        uint32_t mx = 0;
        for (int64_t i = 0; i < last; ++i) mx = std::max(mx, eid[i]);
        IdSet bulk_ids(mx, last), bc_ids(mx, last);
        int64_t prev_id = -1;
        int prev_dim = -1;
        int32_t prev_idx = -1;
        std::string msg;
        for (int64_t i = 0; i < last; ++i) {
            int32_t ri;
            if ((int64_t)ereg[i] == prev_id && edim[i] == prev_dim) {
                ri = prev_idx;
            } else {
                ri = reg.of_element(ereg[i], edim[i], msg);
                if (ri < 0) return fail(e0 + i, "element " + std::to_string(eid[i]) + ": " + msg);
                prev_id = ereg[i], prev_dim = edim[i], prev_idx = ri;
            }
            cls[i] = 2;  // 0 bulk, 1 boundary, 2 dropped (a point in a bulk region)
            if (reg.list[ri].boundary) {
                if (!bc_ids.insert(eid[i])) return fail(e0 + i, "repeated boundary element id " + std::to_string(eid[i]));
                cls[i] = 1;
            } else if (edim[i] > 0) {
                if (!bulk_ids.insert(eid[i])) return fail(e0 + i, "repeated element id " + std::to_string(eid[i]));
                cls[i] = 0;
            }
        }
    }
    if (el_err.row != kNone) return fail(el_err.row, el_err.msg);

    // compaction into bulk and boundary lists, both in file order
    const int nt = omp_get_max_threads();
    std::vector<int64_t> cnt(2 * (nt + 1), 0);
#pragma omp parallel num_threads(nt)
    {
        const int th = omp_get_thread_num();
        const int64_t lo = ne * th / nt, hi = ne * (th + 1) / nt;
        int64_t c0 = 0, c1 = 0;
        for (int64_t i = lo; i < hi; ++i) c0 += cls[i] == 0, c1 += cls[i] == 1;
        cnt[2 * (th + 1)] = c0;
        cnt[2 * (th + 1) + 1] = c1;
#pragma omp barrier
#pragma omp single
        for (int q = 1; q <= nt; ++q) cnt[2 * q] += cnt[2 * (q - 1)], cnt[2 * q + 1] += cnt[2 * (q - 1) + 1];
        // implicit barrier after single
        // the output arrays are zero-filled by their resize: one array per thread
        const int64_t nb = cnt[2 * nt], nc = cnt[2 * nt + 1];
#pragma omp sections
        {
#pragma omp section
            out.m.nodes.resize(4 * nb);
#pragma omp section
            out.el_id.resize(nb);
#pragma omp section
            out.m.dim.resize(nb);
#pragma omp section
            out.el_region.resize(nb);
#pragma omp section
            out.el_partition.resize(nb);
#pragma omp section
            {
                out.m.bc_dim.resize(nc);
                out.m.bc_nodes.resize(4 * nc);
                out.bc_id.resize(nc);
                out.bc_region.resize(nc);
            }
        }
        int64_t p0 = cnt[2 * th], p1 = cnt[2 * th + 1];
        for (int64_t i = lo; i < hi; ++i) {
            if (cls[i] == 0) {
                out.m.dim[p0] = edim[i];
                std::copy(&enodes[4 * i], &enodes[4 * i] + 4, &out.m.nodes[4 * p0]);
                out.el_id[p0] = eid[i];
                out.el_region[p0] = (int32_t)ereg[i];
                out.el_partition[p0] = epart[i];
                ++p0;
            } else if (cls[i] == 1) {
                out.m.bc_dim[p1] = edim[i];
                std::copy(&enodes[4 * i], &enodes[4 * i] + 4, &out.m.bc_nodes[4 * p1]);
                out.bc_id[p1] = eid[i];
                out.bc_region[p1] = (int32_t)ereg[i];
                ++p1;
            }
        }
    }
    out.m.n_el = cnt[2 * nt];
    out.m.n_bc = cnt[2 * nt + 1];
    out.m.n_nodes = nn;
    out.node_id.assign(nid.begin(), nid.end());
    out.from_file = true;
    for (const Region &r : reg.list) {
        out.region_id.push_back(r.id);
        out.region_dim.push_back(r.dim);
        out.region_boundary.push_back(r.boundary ? 1 : 0);
        out.region_name.push_back(r.name);
    }
    for (const std::string &s : out.region_name) out.region_name_ptr.push_back(s.c_str());
    return MH_OK;
}

// GMSH_DataHeader of read_data_header (msh_gmshreader.cc:251-301), from the line after the
// one holding "$ElementData"; k is left on the last header line
struct DataHeader {
    std::string name;
    double time = 0.0;
    uint32_t n_components = 1, n_entities = 0;
};

bool read_header(const Text &t, int64_t &k, DataHeader &h) {
    const int64_t nl = t.n_line;
    auto at = [&](int64_t r) { return r < nl; };
    uint32_t n_str, n_real, n_int, v;
    if (!at(k) || !Line(t, k).u32(n_str)) return false;
    if (n_str > 0) {
        if (!at(++k)) return false;
        h.name = Line(t, k).str();
    }
    k += n_str > 0 ? n_str - 1 : 0;
    if (!at(++k) || !Line(t, k).u32(n_real)) return false;
    if (n_real > 0) {
        if (!at(++k) || !Line(t, k).f64(h.time)) return false;
        k += n_real - 1;
    }
    if (!at(++k) || !Line(t, k).u32(n_int)) return false;
    uint32_t ints[3] = {0, 1, 0};
    for (uint32_t j = 0; j < n_int && j < 3; ++j) {
        if (!at(++k) || !Line(t, k).u32(v)) return false;
        ints[j] = v;
    }
    if (n_int > 3) k += n_int - 3;
    h.n_components = ints[1];
    h.n_entities = ints[2];
    return true;
}

int element_data(const char *path, const char *field, double time, int64_t n_ids, const int64_t *ids,
                 int32_t n_comp, double *out, std::string &err) {
    if (!path || !field || n_ids < 0 || n_comp < 1 || (n_ids > 0 && (!ids || !out))) {
        err = "invalid argument";
        return MH_ERR_INVALID;
    }
    for (int64_t i = 1; i < n_ids; ++i)
        if (ids[i] <= ids[i - 1]) {
            err = "el_ids must be strictly ascending";
            return MH_ERR_INVALID;
        }
    Text t;
    int rc = load(path, t, err);
    if (rc) return rc;
    const int64_t nl = t.n_line;
    std::fill(out, out + n_ids * n_comp, std::numeric_limits<double>::quiet_NaN());
    const double limit = time * (1.0 + 2.0 * std::numeric_limits<double>::epsilon());
    bool found = false, used = false;
    std::vector<int64_t> lb;
    std::vector<uint8_t> state;
    std::vector<double> vals;
    for (int64_t k = 0; k < nl;) {
        k = skip_to(t, k, "$ElementData");
        if (k == kNone) break;
        int64_t h0 = k + 1;
        DataHeader h;
        if (!read_header(t, h0, h)) {
            err = t.where(std::min(h0, nl)) + ": wrong format of the $ElementData header";
            return MH_ERR_INVALID;
        }
        k = h0 + 1;
        if (h.name != field) continue;
        found = true;
        if (h.time > limit) break;
        used = true;
        const int64_t rows = std::min<int64_t>(h.n_entities, nl - k);
        // Per row, in parallel: the first index of ids not below the row's id and, when that
        // id is the row's, its values.  A row is stored iff the forward-only pointer of the
        // ordered pass stops at exactly that index.
        lb.assign(rows, 0);
        state.assign(rows, 0);  // 0 id unreadable, 1 no match, 2 values read, 3 values unreadable
        vals.resize((size_t)rows * n_comp);
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < rows; ++r) {
            Line l(t, k + r);
            uint32_t id;
            if (!l.u32(id)) continue;
            lb[r] = std::lower_bound(ids, ids + n_ids, (int64_t)id) - ids;
            state[r] = 1;
            if (lb[r] == n_ids || ids[lb[r]] != (int64_t)id) continue;
            state[r] = 2;
            for (int32_t c = 0; c < n_comp; ++c)
                if (!l.f64(vals[(size_t)r * n_comp + c])) {
                    state[r] = 3;
                    break;
                }
        }
        int64_t pos = 0;
        for (int64_t r = 0; r < rows; ++r) {
            if (state[r] == 0) {
                err = t.where(k + r) + ": wrong format of $ElementData line";
                return MH_ERR_INVALID;
            }
            pos = std::max(pos, lb[r]);
            if (pos == n_ids) break;  // an id past the last element: the rest is skipped
            if (state[r] == 1 || pos != lb[r]) continue;
            if (state[r] == 3) {
                err = t.where(k + r) + ": element " + std::to_string(ids[pos]) + " of field '" + field +
                      "' has fewer than " + std::to_string(n_comp) + " values or a malformed one";
                return MH_ERR_INVALID;
            }
            std::copy(&vals[(size_t)r * n_comp], &vals[(size_t)r * n_comp] + n_comp, out + pos * n_comp);
        }
        if (h.n_entities > (uint32_t)rows) break;  // the file ended inside the section
        k += rows;
    }
    if (!found) {
        err = t.path + ": no $ElementData section for field '" + field + "'";
        return MH_ERR_INVALID;
    }
    if (!used) {
        err = t.path + ": no $ElementData of field '" + field + "' at or before time " + std::to_string(time);
        return MH_ERR_INVALID;
    }
    return MH_OK;
}

void copy_err(const std::string &msg, char *err, size_t len) {
    if (!err || len == 0) return;
    const size_t n = std::min(msg.size(), len - 1);
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

}  // namespace

extern "C" {

int mh_gmsh_read(const char *path, mh_mesh **out, char *err, size_t err_len) {
    copy_err("", err, err_len);
    if (!path || !out) {
        copy_err("invalid argument", err, err_len);
        return MH_ERR_INVALID;
    }
    *out = nullptr;
    std::unique_ptr<mh_mesh> m(new (std::nothrow) mh_mesh());
    if (!m) return MH_ERR_NOMEM;
    std::string msg;
    int rc;
    try {
        rc = read_mesh(path, *m, msg);
    } catch (const std::bad_alloc &) {
        rc = MH_ERR_NOMEM;
        msg = "out of host memory reading '" + std::string(path) + "'";
    }
    if (rc) {
        copy_err(msg, err, err_len);
        return rc;
    }
    *out = m.release();
    return MH_OK;
}

int mh_gmsh_info_get(const mh_mesh *m, mh_gmsh_info *info) {
    if (!m || !info || !m->from_file) return MH_ERR_INVALID;
    info->node_id = m->node_id.data();
    info->el_id = m->el_id.data();
    info->el_region = m->el_region.data();
    info->el_partition = m->el_partition.data();
    info->bc_id = m->bc_id.data();
    info->bc_region = m->bc_region.data();
    info->n_regions = (int32_t)m->region_id.size();
    info->region_id = m->region_id.data();
    info->region_dim = m->region_dim.data();
    info->region_boundary = m->region_boundary.data();
    info->region_name = m->region_name_ptr.data();
    return MH_OK;
}

int mh_gmsh_element_data(const char *path, const char *field, double time, int64_t n_ids, const int64_t *el_ids,
                         int32_t n_components, double *out, char *err, size_t err_len) {
    copy_err("", err, err_len);
    std::string msg;
    int rc;
    try {
        rc = element_data(path, field, time, n_ids, el_ids, n_components, out, msg);
    } catch (const std::bad_alloc &) {
        rc = MH_ERR_NOMEM;
        msg = "out of host memory";
    }
    copy_err(msg, err, err_len);
    return rc;
}

}  // extern "C"
