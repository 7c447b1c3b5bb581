// g3x_synth.cpp -- seeded synthetic workloads for the extension benchmarks and tests.
//
// Host-only utility library (libg3x_synth.so).  It produces extension jobs in the shapes
// of the benchmark configurations; the reference's own datasets are not used.  Output:
//   u8[]    one byte per base (0-3, 4 = N); a job's query/target are u8[off .. off+len)
//   jobs[]  g3x_job_t records whose q_off/t_off are those same base indices, so packing u8[]
//           into the 2-bit/N planes at base 0 gives the device stream directly
//   seeds[] (kind 2 only) one record per seed for the left/right band-retry driver
//
// Kinds:
//   1  right-extension jobs: query length U[1,150], N at 0.1%; target = query with 1%
//      substitutions and 0.1% indels (geometric length, mean 2) + w random flank bases;
//      h0 U[19,150].  A fraction `unrelated` of jobs (0 for the config-1 workload) gets a
//      random target of the query's length instead of the mutated copy.
//   2  seeds on reads of 100/150/250 bp (equal mix): seed start uniform over the read,
//      length U[19,50]; per-seed divergence U[0,5%] (90% substitutions, 10% indel events of
//      geometric length, mean 2); a fraction `unrelated` of seeds gets random flanks.  The
//      reference window around the seed is [rmax0, rmax1) exactly as mem_chain2aln computes
//      it for a one-seed chain (bwa/src/aux.cu:187-205 with cal_max_gap, aux.cu:168-175).
//      Jobs: the left extension (reversed read prefix vs reversed window prefix, read
//      through the QREV/TREV flags) and the right extension, both with h0 = len * a.
//   4  long segments: query length log-uniform [500,5000], divergence U[0.1%,1%] (90%
//      substitutions, 10% indel events of length U[1,20]); target = mutated query +
//      min(cal_max_gap(qlen), 2w) random flank bases; h0 U[19,150].
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <algorithm>
#include <thread>
#include <vector>
#include "../../include/g3x.h"

namespace {

struct Rng {   // splitmix64 stream
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    int range(int lo, int hi) { return lo + (int)(next() % (uint64_t)(hi - lo + 1)); }  // [lo, hi]
    int base() { return (int)(next() & 3); }
    int geom_half() { int L = 1; while (uni() < 0.5) ++L; return L; }                  // mean 2
};

struct Params {
    int32_t kind, n, w, a, o_del, e_del, o_ins, e_ins, threads;
    double unrelated;
    uint64_t seed;
};

int cal_max_gap(const Params& p, int qlen) {   // bwa/src/aux.cu:168-175
    int l_del = (int)((double)(qlen * p.a - p.o_del) / p.e_del + 1.);
    int l_ins = (int)((double)(qlen * p.a - p.o_ins) / p.e_ins + 1.);
    int l = l_del > l_ins ? l_del : l_ins;
    l = l > 1 ? l : 1;
    return l < p.w << 1 ? l : p.w << 1;
}

// Copies src with substitutions and indel events.  indel_len: 0 = geometric mean 2,
// otherwise uniform [1, indel_len].
void mutate(Rng& g, const uint8_t* src, int n, double psub, double pindel, int indel_len,
            std::vector<uint8_t>& out) {
    for (int k = 0; k < n;) {
        if (pindel > 0 && g.uni() < pindel) {
            int L = indel_len ? g.range(1, indel_len) : g.geom_half();
            if (g.next() & 1) {
                for (int t = 0; t < L; ++t) out.push_back((uint8_t)g.base());
            } else {
                k += L;
                continue;
            }
        }
        uint8_t b = src[k++];
        if (b < 4 && psub > 0 && g.uni() < psub) b = (uint8_t)((b + 1 + (g.next() % 3)) & 3);
        out.push_back(b);
    }
}

void random_seq(Rng& g, int n, double pn, std::vector<uint8_t>& out) {
    for (int k = 0; k < n; ++k) out.push_back(pn > 0 && g.uni() < pn ? 4 : (uint8_t)g.base());
}

struct SeedRec {   // mirrors the oracle's g3o_seed
    int64_t read_off, win_off, rmax0, rmax1, rbeg;
    int32_t l_query, qbeg, len;
    int32_t pad_;
};

struct Chunk {
    std::vector<uint8_t> u8;
    std::vector<g3x_job_t> jobs;
    std::vector<SeedRec> seeds;
};

void gen_unit(const Params& p, int64_t idx, Chunk& ch) {
    Rng g(p.seed * 0x2545F4914F6CDD1Dull + (uint64_t)idx * 0x9E3779B97F4A7C15ull + 0x6A5);
    g.next();
    const uint32_t base0 = (uint32_t)ch.u8.size();
    if (p.kind == 1 || p.kind == 4) {
        int qlen;
        double psub, pind;
        int indel_len, flank;
        if (p.kind == 1) {
            qlen = g.range(1, 150); psub = 0.01; pind = 0.001; indel_len = 0; flank = p.w;
        } else {
            qlen = (int)floor(exp(log(500.0) + g.uni() * (log(5000.0) - log(500.0))));
            double d = 0.001 + g.uni() * 0.009;
            psub = 0.9 * d; pind = 0.1 * d; indel_len = 20;
            flank = cal_max_gap(p, qlen);
        }
        random_seq(g, qlen, 0.001, ch.u8);
        std::vector<uint8_t> t;
        if (p.kind == 1 && p.unrelated > 0 && g.uni() < p.unrelated) {
            random_seq(g, qlen, 0.0, t);                 // unrelated target
        } else {
            mutate(g, ch.u8.data() + base0, qlen, psub, pind, indel_len, t);
        }
        random_seq(g, flank, 0.0, t);
        if (t.size() > 65535) t.resize(65535);
        const uint32_t toff = (uint32_t)ch.u8.size();
        ch.u8.insert(ch.u8.end(), t.begin(), t.end());
        g3x_job_t jb;
        jb.q_off = base0; jb.t_off = toff; jb.qlen = (uint16_t)qlen; jb.tlen = (uint16_t)t.size();
        jb.h0 = g.range(19, 150); jb.w = p.w; jb.flags = 0;
        ch.jobs.push_back(jb);
        return;
    }
    // kind 2: one seed on one read
    static const int kLens[3] = {100, 150, 250};
    const int L = kLens[g.next() % 3];
    const int len = g.range(19, 50);
    const int qbeg = g.range(0, L - len);
    const int qe = qbeg + len;
    const double d = g.uni() * 0.05;
    const bool unrelated = g.uni() < p.unrelated;
    random_seq(g, L, 0.001, ch.u8);
    const uint8_t* read = nullptr;
    std::vector<uint8_t> rd(ch.u8.begin() + base0, ch.u8.end());
    read = rd.data();
    const int gl = cal_max_gap(p, qbeg), gr = cal_max_gap(p, L - qe);
    const int64_t rbeg = 1000000;                       // arbitrary reference coordinate
    const int64_t rmax0 = rbeg - (qbeg + gl);            // aux.cu:192-193 for a 1-seed chain
    const int64_t rmax1 = rbeg + len + ((L - qe) + gr);  // aux.cu:194
    const int left_len = (int)(rbeg - rmax0), right_len = (int)(rmax1 - (rbeg + len));
    // left reference part, ending at rbeg: related = mutated read prefix, left-padded
    std::vector<uint8_t> left, right;
    if (!unrelated) {
        std::vector<uint8_t> m;
        mutate(g, read, qbeg, 0.9 * d, 0.1 * d, 0, m);
        if ((int)m.size() > left_len) m.erase(m.begin(), m.begin() + ((int)m.size() - left_len));
        random_seq(g, left_len - (int)m.size(), 0.0, left);
        left.insert(left.end(), m.begin(), m.end());
        mutate(g, read + qe, L - qe, 0.9 * d, 0.1 * d, 0, right);
        if ((int)right.size() > right_len) right.resize(right_len);
        random_seq(g, right_len - (int)right.size(), 0.0, right);
    } else {
        random_seq(g, left_len, 0.0, left);
        random_seq(g, right_len, 0.0, right);
    }
    const uint32_t woff = (uint32_t)ch.u8.size();
    ch.u8.insert(ch.u8.end(), left.begin(), left.end());
    ch.u8.insert(ch.u8.end(), read + qbeg, read + qe);   // the seed is an exact match
    ch.u8.insert(ch.u8.end(), right.begin(), right.end());
    SeedRec s;
    s.read_off = base0; s.win_off = woff; s.rmax0 = rmax0; s.rmax1 = rmax1; s.rbeg = rbeg;
    s.l_query = L; s.qbeg = qbeg; s.len = len; s.pad_ = 0;
    ch.seeds.push_back(s);
    if (qbeg > 0) {
        g3x_job_t jb;
        jb.q_off = base0; jb.qlen = (uint16_t)qbeg;
        jb.t_off = woff; jb.tlen = (uint16_t)left_len;
        jb.h0 = len * p.a; jb.w = p.w; jb.flags = G3X_JOB_QREV | G3X_JOB_TREV;
        ch.jobs.push_back(jb);
    }
    if (qe != L) {
        g3x_job_t jb;
        jb.q_off = base0 + (uint32_t)qe; jb.qlen = (uint16_t)(L - qe);
        jb.t_off = woff + (uint32_t)(left_len + len); jb.tlen = (uint16_t)right_len;
        jb.h0 = len * p.a; jb.w = p.w; jb.flags = 0;
        ch.jobs.push_back(jb);
    }
}

struct Synth {
    std::vector<uint8_t> u8;
    std::vector<g3x_job_t> jobs;
    std::vector<SeedRec> seeds;
};

}  // namespace

extern "C" {

typedef struct {
    int32_t kind, n, w, a, o_del, e_del, o_ins, e_ins, threads, pad_;
    double unrelated;
    uint64_t seed;
} g3x_synth_params_t;

void* g3x_synth_create(const g3x_synth_params_t* ps) {
    if (!ps || ps->n < 0 || (ps->kind != 1 && ps->kind != 2 && ps->kind != 4)) return nullptr;
    Params p;
    p.kind = ps->kind; p.n = ps->n; p.w = ps->w; p.a = ps->a; p.o_del = ps->o_del;
    p.e_del = ps->e_del; p.o_ins = ps->o_ins; p.e_ins = ps->e_ins; p.unrelated = ps->unrelated;
    p.seed = ps->seed;
    int T = ps->threads > 0 ? ps->threads : (int)std::thread::hardware_concurrency();
    if (T < 1) T = 1;
    T = std::min<int>(T, std::max<int>(1, p.n / 1024));
    std::vector<Chunk> chunks((size_t)T);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) {
        pool.emplace_back([&, t]() {
            int64_t b = (int64_t)p.n * t / T, e = (int64_t)p.n * (t + 1) / T;
            for (int64_t k = b; k < e; ++k) gen_unit(p, k, chunks[t]);
        });
    }
    for (auto& th : pool) th.join();
    Synth* s = new Synth();
    size_t nb = 0, nj = 0, ns = 0;
    for (auto& c : chunks) { nb += c.u8.size(); nj += c.jobs.size(); ns += c.seeds.size(); }
    s->u8.reserve(nb); s->jobs.reserve(nj); s->seeds.reserve(ns);
    for (auto& c : chunks) {
        uint32_t shift = (uint32_t)s->u8.size();
        s->u8.insert(s->u8.end(), c.u8.begin(), c.u8.end());
        for (auto jb : c.jobs) { jb.q_off += shift; jb.t_off += shift; s->jobs.push_back(jb); }
        for (auto sd : c.seeds) { sd.read_off += shift; sd.win_off += shift; s->seeds.push_back(sd); }
    }
    return s;
}

int64_t g3x_synth_count(void* h, int what) {
    Synth* s = static_cast<Synth*>(h);
    if (!s) return -1;
    return what == 0 ? (int64_t)s->jobs.size() : what == 1 ? (int64_t)s->u8.size() : (int64_t)s->seeds.size();
}

int g3x_synth_copy(void* h, g3x_job_t* jobs, uint8_t* u8, void* seeds) {
    Synth* s = static_cast<Synth*>(h);
    if (!s) return -1;
    if (jobs && !s->jobs.empty()) memcpy(jobs, s->jobs.data(), s->jobs.size() * sizeof(g3x_job_t));
    if (u8 && !s->u8.empty()) memcpy(u8, s->u8.data(), s->u8.size());
    if (seeds && !s->seeds.empty()) memcpy(seeds, s->seeds.data(), s->seeds.size() * sizeof(SeedRec));
    return 0;
}

void g3x_synth_free(void* h) { delete static_cast<Synth*>(h); }

// Packs u8 codes into the 2-bit/N planes (base index = byte index), multi-threaded.
// codes needs ceil(n/16) words, nmask ceil(n/32) words.
int g3x_synth_pack(const uint8_t* u8, int64_t n, uint32_t* codes, uint32_t* nmask, int threads) {
    if (n < 0) return -1;
    int64_t words = (n + 31) / 32;
    int T = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (T < 1) T = 1;
    auto work = [&](int64_t wb, int64_t we) {
        for (int64_t wd = wb; wd < we; ++wd) {
            uint32_t c0 = 0, c1 = 0, nm = 0;
            int64_t b0 = wd * 32;
            for (int k = 0; k < 32; ++k) {
                int64_t b = b0 + k;
                uint32_t v = b < n ? u8[b] : 0u;
                uint32_t c = v & 3u;
                if (v > 3) nm |= 1u << k;
                if (k < 16) c0 |= c << (2 * k); else c1 |= c << (2 * (k - 16));
            }
            codes[2 * wd] = c0;
            if (2 * wd + 1 < (n + 15) / 16) codes[2 * wd + 1] = c1;
            nmask[wd] = nm;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) pool.emplace_back(work, words * t / T, words * (t + 1) / T);
    for (auto& th : pool) th.join();
    return 0;
}

}  // extern "C"
