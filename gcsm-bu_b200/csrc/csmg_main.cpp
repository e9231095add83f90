// csmg: command-line drop-in for the reference's `csmg` (main.cpp:162-190), built on libcsm.
//
// Flags, defaults and boolean parsing follow utils/simple_command_parser.h:13-76 and
// utils/technique_option.h:58-86; file formats follow graph/graph.cpp:191-563 (`t` lines
// skipped, `v id label`, `e src dst label`).  The update file may also carry `-e src dst label`
// lines (deletions), an extension the reference does not read.  The lines the reference's
// experiment scripts parse are printed verbatim (technique_permutation.h:129-130, :224 and
// the PRINT_LOCAL_TIME format of utils/cuda_helpers.h:96-100).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/csm.h"

namespace {

struct Args {
    std::vector<std::string> tok;
    std::string get(const std::string &o) const {
        for (size_t i = 0; i + 1 < tok.size(); i++)
            if (tok[i] == o) return tok[i + 1];
        return "";
    }
    int32_t get_i32(const std::string &o, int32_t def) const {
        std::string v = get(o);
        return v.empty() ? def : (int32_t)std::stol(v);
    }
    uint32_t get_u32(const std::string &o, uint32_t def) const {
        std::string v = get(o);
        return v.empty() ? def : (uint32_t)std::stoul(v);
    }
    bool get_bool(const std::string &o, bool def) const {
        std::string v = get(o);
        if (v == "true" || v == "True") return true;
        if (v == "false" || v == "False") return false;
        return def;
    }
};

bool read_file(const std::string &path, std::string &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    out.resize(got);
    return true;
}

// Whitespace tokenizer over a text buffer.
struct Scanner {
    const char *p, *e;
    explicit Scanner(const std::string &s) : p(s.data()), e(s.data() + s.size()) {}
    void skip() {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    }
    bool word(std::string &w) {
        skip();
        if (p >= e) return false;
        const char *b = p;
        while (p < e && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
        w.assign(b, p);
        return true;
    }
    bool num(uint64_t &v) {
        skip();
        if (p >= e || *p < '0' || *p > '9') return false;
        v = 0;
        while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (uint64_t)(*p++ - '0');
        return true;
    }
};

struct TextGraph {
    std::vector<uint32_t> vlabel;  // UINT32_MAX = absent
    std::vector<uint32_t> src, dst, elab;
};

bool load_graph_text(const std::string &path, TextGraph &g, bool is_query) {
    std::string buf;
    if (!read_file(path, buf)) return false;
    Scanner sc(buf);
    std::string w;
    uint64_t a, b, c;
    while (sc.word(w)) {
        if (w == "t") {
            sc.word(w);
            sc.num(a);
        } else if (w == "v") {
            if (!sc.num(a) || !sc.num(b)) break;
            if (a >= g.vlabel.size()) g.vlabel.resize(a + 1, UINT32_MAX);
            if (g.vlabel[a] == UINT32_MAX) g.vlabel[a] = (uint32_t)b;
        } else {
            if (!sc.num(a) || !sc.num(b) || !sc.num(c)) break;
            g.src.push_back((uint32_t)a);
            g.dst.push_back((uint32_t)b);
            g.elab.push_back((uint32_t)c);
        }
    }
    (void)is_query;
    return true;
}

// Binary data graph (magic "CSMBGRF1"): u32 nv, u32 0, u64 ne, u32 vlabel[nv], u32 src[ne],
// u32 dst[ne], u32 elabel[ne], little-endian.  Returns false if `buf` is not one.
bool load_graph_binary(const std::string &buf, TextGraph &g, bool &ok) {
    ok = false;
    if (buf.size() < 24 || buf.compare(0, 8, "CSMBGRF1") != 0) return false;
    uint32_t nv = 0;
    uint64_t ne = 0;
    std::memcpy(&nv, buf.data() + 8, 4);
    std::memcpy(&ne, buf.data() + 16, 8);
    if (buf.size() != 24 + 4ull * nv + 12ull * ne) return true;
    const char *p = buf.data() + 24;
    g.vlabel.resize(nv);
    std::memcpy(g.vlabel.data(), p, 4ull * nv);
    p += 4ull * nv;
    for (auto *v : {&g.src, &g.dst, &g.elab}) {
        v->resize(ne);
        std::memcpy(v->data(), p, 4 * ne);
        p += 4 * ne;
    }
    ok = true;
    return true;
}

void print_info(const Args &args, const std::string &q, const std::string &d, const std::string &u, int32_t dev,
                uint32_t bs, bool show_mem, const csm_config &cfg) {
    static const char *orders[] = {"BFS Order", "Gamma Order", "RapidCSM Order", "RI Order"};
    static const char *strategies[] = {"DFS w/ Work Stealing", "DFS w/o Work Stealing", "Dynamic BFS DFS", "BFS"};
    int mo = cfg.matching_order, ss = cfg.search_strategy, li = cfg.local_index, cp = cfg.cartesian_product,
        hv = cfg.heavy_vertex_avoidance, rs = cfg.relation_switch;
    switch (cfg.algorithm) {  // presets of utils/technique_option.h:60-71
        case 1: mo = 2; ss = 2; li = 1; cp = 1; hv = 1; rs = 1; break;
        case 2: mo = 1; ss = 0; li = 0; cp = 1; hv = 0; rs = 0; break;
        case 4: mo = 0; ss = 2; li = 0; cp = 1; hv = 1; rs = 1; break;
        case 5: mo = 1; ss = 2; li = 0; cp = 1; hv = 1; rs = 1; break;
        default: break;
    }
    (void)args;
    std::cout << "--------------------------------------------------------------------" << std::endl;
    std::cout << "Command Line:\n\tQuery Graph: " << q << "\n\tData Graph: " << d << "\n\tData Graph Update: " << u
              << "\n\tDevice ID: " << dev << "\n\tBatch Size: " << bs << "\n\tShow GPU Memory?: " << (show_mem ? "yes" : "no")
              << '\n';
    std::cout << "--------------------------------------------------------------------" << std::endl;
    std::cout << "Technique Option:\n\tMatching Order: " << orders[mo & 3] << "\n\tSearch Strategy: " << strategies[ss & 3]
              << "\n\tUse Local Index?: " << (li ? "w/ Local Index" : "w/o Local Index")
              << "\n\tUse Cartesian Product?: " << (cp ? "w/ Cartesian Product" : "w/o Use Cartesian Product")
              << "\n\tUse Heavy Vertex Avoidance?: " << (hv ? "w/ Heavy Vertex Avoidance" : "w/o Use Heavy Vertex Avoidance")
              << "\n\tUse Relation Switch?: " << (rs ? "w/ Relation Switch" : "w/o Use Relation Switch") << '\n';
    std::cout << "--------------------------------------------------------------------" << std::endl;
    std::cout << "Engine: " << csm_version() << '\n';
    std::cout << "--------------------------------------------------------------------" << std::endl;
}

void print_time(const char *name, double host_ms, double kernel_ms) {
    std::cout << name << ", time (ms): " << (unsigned long)host_ms << "(host), " << (unsigned long)kernel_ms << "(kernel)\n";
}

int die(csm_engine *e, const char *what) {
    char buf[512];
    csm_last_error(e, buf, sizeof buf);
    std::cout << what << ": " << buf << std::endl;
    if (e) csm_destroy(e);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    Args args;
    for (int i = 1; i < argc; i++) args.tok.emplace_back(argv[i]);
    std::string cmd = "csmg";
    for (auto &t : args.tok) cmd += " " + t;
    std::cout << cmd << std::endl;

    const std::string qpath = args.get("--query"), dpath = args.get("--data"), upath = args.get("--update");
    const int32_t device = args.get_i32("--device", 0);
    const uint32_t batch_size = args.get_u32("--batch_size", UINT32_MAX);
    const int32_t algorithm = args.get_i32("--algorithm", 0);
    const bool show_mem = args.get_bool("--show_gpu_memory", false);
    const bool print_indexing = args.get_bool("--print_indexing_time", false);

    csm_config cfg;
    csm_default_config(&cfg);
    cfg.device = device;
    cfg.algorithm = algorithm;
    cfg.matching_order = args.get_i32("--matching_order", 2);
    cfg.search_strategy = args.get_i32("--search_strategy", 2);
    cfg.local_index = args.get_bool("--local_index", true);
    cfg.cartesian_product = args.get_bool("--cartesian_product", true);
    cfg.heavy_vertex_avoidance = args.get_bool("--heavy_vertex_avoidance", true);
    cfg.relation_switch = args.get_bool("--relation_switch", true);
    const std::string mat = args.get("--materialize_rows");
    if (!mat.empty()) cfg.materialize_rows = std::stoull(mat);
    print_info(args, qpath, dpath, upath, device, batch_size, show_mem, cfg);

    std::cout << "----------- Read Graphs from Files ------------\n";
    auto t0 = std::chrono::high_resolution_clock::now();
    TextGraph qg, dg;
    if (!load_graph_text(qpath, qg, true)) {
        std::cout << "Failed to open: " << qpath << std::endl;
        return 255;
    }
    // Extensions: --snapshot_in restores a device-state checkpoint instead of reading --data;
    // --snapshot_out writes one after the stream.  Data and update files may be binary.
    const std::string snap_in = args.get("--snapshot_in"), snap_out = args.get("--snapshot_out");
    if (snap_in.empty()) {
        std::string dbuf;
        if (!read_file(dpath, dbuf)) {
            std::cout << "Failed to open: " << dpath << std::endl;
            return 255;
        }
        bool bin_ok = false;
        if (load_graph_binary(dbuf, dg, bin_ok)) {
            if (!bin_ok) {
                std::cout << "Corrupt binary data graph: " << dpath << std::endl;
                return 255;
            }
        } else if (!load_graph_text(dpath, dg, false)) {
            std::cout << "Failed to open: " << dpath << std::endl;
            return 255;
        }
    }
    // Update stream: batch k = update lines [k*B, (k+1)*B), counting every update line
    // (graph.cpp:507-516), filtered or not.
    std::string ubuf;
    if (!read_file(upath, ubuf)) {
        std::cout << "Failed to open: " << upath << std::endl;
        return 255;
    }
    struct Batch {
        std::vector<uint32_t> src, dst, lab;
        std::vector<uint8_t> del;
        bool any_del = false;
    };
    std::vector<Batch> batches;
    if (ubuf.size() >= 16 && ubuf.compare(0, 8, "CSMBUPD1") == 0) {
        // Binary update stream: u64 n, u32 src[n], u32 dst[n], u32 elabel[n], u8 is_delete[n].
        uint64_t n = 0;
        std::memcpy(&n, ubuf.data() + 8, 8);
        if (ubuf.size() != 16 + 13 * n || batch_size == 0) {
            std::cout << "Corrupt binary update stream: " << upath << std::endl;
            return 255;
        }
        const uint32_t *us = reinterpret_cast<const uint32_t *>(ubuf.data() + 16);
        const uint32_t *ud = us + n, *ul = ud + n;
        const uint8_t *udel = reinterpret_cast<const uint8_t *>(ul + n);
        for (uint64_t i = 0; i < n; i++) {
            if (i % batch_size == 0) batches.emplace_back();
            Batch &bt = batches.back();
            bt.src.push_back(us[i]);
            bt.dst.push_back(ud[i]);
            bt.lab.push_back(ul[i]);
            bt.del.push_back(udel[i] ? 1 : 0);
            bt.any_del |= udel[i] != 0;
        }
    } else {
        Scanner sc(ubuf);
        std::string w;
        uint64_t a, b, c, nlines = 0;
        while (sc.word(w)) {
            if (w == "t") {
                sc.word(w);
                sc.num(a);
                continue;
            }
            if (w == "v") {
                std::cout << "vertex update.\n";
                return 255;
            }
            if (!sc.num(a) || !sc.num(b) || !sc.num(c)) break;
            if (batch_size == 0) {
                std::cout << "batch size must be positive\n";
                return 255;
            }
            if (nlines % batch_size == 0) batches.emplace_back();
            nlines++;
            Batch &bt = batches.back();
            bt.src.push_back((uint32_t)a);
            bt.dst.push_back((uint32_t)b);
            bt.lab.push_back((uint32_t)c);
            const bool del = w == "-e";
            bt.del.push_back(del ? 1 : 0);
            bt.any_del |= del;
        }
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    print_time("Read Graphs from Files", std::chrono::duration<double, std::milli>(t1 - t0).count(), 0);

    if (qg.vlabel.size() < 2) {
        std::cout << "the number of query verticex should not be less than 2!" << std::endl;
        return 255;
    }
    std::cout << "----------- Preprocessing ------------\n";
    csm_engine *e = nullptr;
    if (csm_create(&e, &cfg) != CSM_OK) return die(nullptr, "csm_create");
    int32_t qid = -1;
    if (csm_load_query(e, (uint32_t)qg.vlabel.size(), qg.vlabel.data(), (uint32_t)qg.src.size(), qg.src.data(),
                       qg.dst.data(), qg.elab.data(), &qid) != CSM_OK)
        return die(e, "query");
    t0 = std::chrono::high_resolution_clock::now();
    if (!snap_in.empty()) {
        if (csm_load_snapshot(e, snap_in.c_str()) != CSM_OK) return die(e, "snapshot");
    } else {
        if (csm_load_graph(e, (uint32_t)dg.vlabel.size(), dg.vlabel.data(), dg.src.size(), dg.src.data(),
                           dg.dst.data(), dg.elab.data()) != CSM_OK)
            return die(e, "data graph");
        std::cout << "#data graph vertices: " << dg.vlabel.size() << std::endl;
    }
    t1 = std::chrono::high_resolution_clock::now();
    print_time("Build Global Index Offline", std::chrono::duration<double, std::milli>(t1 - t0).count(), 0);
    {
        std::string plan(1 << 16, '\0');
        csm_describe_plan(e, qid, &plan[0], plan.size());
        std::cout << plan.c_str();
    }
    if (show_mem) {
        uint64_t fr = 0, tot = 0;
        csm_device_memory(e, &fr, &tot);
        std::cout << "Total GPU memory: " << tot / 1024 / 1024 << " MiB\nFree GPU memory: " << fr / 1024 / 1024 << " MiB"
                  << std::endl;
    }

    std::cout << "--------- Incremental Matching --------\n";
    unsigned long long num_pos = 0, num_neg = 0;
    double kernel_ms = 0;
    t0 = std::chrono::high_resolution_clock::now();
    for (size_t k = 0; k < batches.size(); k++) {
        Batch &bt = batches[k];
        std::cout << std::endl << "Batch #" << k << " --------" << std::endl;
        csm_batch_result r;
        auto b0 = std::chrono::high_resolution_clock::now();
        if (csm_apply_batch(e, bt.src.size(), bt.src.data(), bt.dst.data(), bt.lab.data(),
                            bt.any_del ? bt.del.data() : nullptr, &r) != CSM_OK)
            return die(e, "batch");
        auto b1 = std::chrono::high_resolution_clock::now();
        num_pos += r.positive;
        num_neg += r.negative;
        kernel_ms += r.latency_ns / 1e6;
        if (print_indexing)
            std::cout << "Finish Index Maintenance, time (ms): " << (unsigned long)(r.apply_ns / 1e6) << "(host), "
                      << (unsigned long)(r.apply_ns / 1e6) << "(kernel)\n";
        std::cout << "Batch #" << k << ": pos=" << r.positive << " neg=" << r.negative << " ins=" << r.inserted
                  << " del=" << r.deleted << " lat_us=" << (unsigned long long)(r.latency_ns / 1000)
                  << " host_us=" << (unsigned long long)std::chrono::duration<double, std::micro>(b1 - b0).count()
                  << std::endl;
    }
    t1 = std::chrono::high_resolution_clock::now();
    print_time("Incremental Matching", std::chrono::duration<double, std::milli>(t1 - t0).count(), kernel_ms);
    std::cout << "--------------------------------------------------------------------" << std::endl;
    std::cout << "Num Positive Matches: " << num_pos << '\n';
    std::cout << "Num Negative Matches: " << num_neg << '\n';
    if (!snap_out.empty() && csm_save_snapshot(e, snap_out.c_str()) != CSM_OK) return die(e, "snapshot");
    csm_destroy(e);
    return 0;
}
