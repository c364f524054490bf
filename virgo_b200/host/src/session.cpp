// Whole proofs without the reference verifier in the loop.
//
// The protocol is interactive, but every verifier challenge comes from the
// same glibc rand() stream as the prover's masks and never depends on a
// prover message.  A session therefore replays the verifier's draws in the
// reference's order (src/linear_gkr/zk_verifier.cpp:910-1253 and
// src/VPD/vpd_verifier.cpp:80-335) and calls the prover exactly as the
// verifier would, producing the same messages, roots and query answers.
// The verifier's own checks and its predicate evaluation are not run; the
// one prover input that comes from the predicates, the general value of
// sumcheck_finalround (zk_verifier.cpp:1149), is fixed by the sumcheck claim
// itself: finalround(0) + finalround(1) + direct_relay * v_u must equal the
// running claim, and the general value enters finalround's linear
// coefficient only, so it is that difference.
//
// The transcript has the record layout of the oracle's recorder: 1 byte tag,
// uint32 count of 16-byte units, the units.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <algorithm>
#include <memory>
#include <thread>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "device.h"
#include "internal.h"
#include "linear_gkr/zk_prover.h"
#include "poly_commitment/poly_commit.h"

typedef prime_field::field_element F;
using clk = std::chrono::high_resolution_clock;

int vg_fail(int code, const char *fmt, ...);   // sets vg_last_error()

static double since(clk::time_point t0)
{
    return std::chrono::duration_cast<std::chrono::duration<double>>(clk::now() - t0).count();
}

namespace
{
struct Transcript {
    std::vector<uint8_t> bytes;
    bool on = true;
    void put(char tag, const void *units, uint32_t n16)
    {
        if (!on) return;
        size_t o = bytes.size();
        bytes.resize(o + 5 + 16 * (size_t)n16);
        bytes[o] = (uint8_t)tag;
        memcpy(&bytes[o + 1], &n16, 4);
        if (n16) memcpy(&bytes[o + 5], units, 16 * (size_t)n16);
    }
    void fe(char tag, const F &x) { put(tag, &x, 1); }
    void answer(char tag, const std::pair<std::vector<std::pair<F, F> >, std::vector<__hhash_digest> > &a, int new_size)
    {
        std::vector<uint8_t> buf(16 + a.first.size() * 32 + a.second.size() * 32);
        int64_t hdr[2] = {(int64_t)new_size, (int64_t)((a.first.size() << 16) | a.second.size())};
        memcpy(buf.data(), hdr, 16);
        size_t off = 16;
        for (auto &pv : a.first) {
            memcpy(&buf[off], &pv.first, 16);
            memcpy(&buf[off + 16], &pv.second, 16);
            off += 32;
        }
        for (auto &h : a.second) {
            memcpy(&buf[off], &h, 32);
            off += 32;
        }
        put(tag, buf.data(), (uint32_t)(buf.size() / 16));
    }
};

std::vector<F> draws(int n)
{
    std::vector<F> r(n);
    for (int i = 0; i < n; ++i) r[i] = prime_field::random();
    return r;
}

// zk_verifier.cpp:608-619
F direct_relay(const layered_circuit &C, int depth, const F *r_g, const F *r_u)
{
    if (depth != 1) return F(0);
    F ret(1);
    for (int i = 0; i < C.circuit[depth].bit_length; ++i)
        ret = ret * (F(1) - r_g[i] - r_u[i] + F(2) * r_g[i] * r_u[i]);
    return ret;
}
}  // namespace

// A device circuit and its layer widths, shared by forked sessions.
struct CircuitData {
    layered_circuit C;   // widths only (gates stay on the device)
    vg_circuit *dev = nullptr;
    ~CircuitData()
    {
        if (dev) vg_circuit_destroy(dev);
        delete[] C.circuit;
    }
};

// A session owns its context (CUDA stream, scratch), its commitment state and
// its prover tables, so sessions prove concurrently from different threads.
// Device results of the launch pass, read by the replay pass.
struct PassResults {
    const F *rec = nullptr;   // GKR records (9 values each)
    int nrec = 0;
    vg_pc_results pc{};
    int levels = 0;
    // the replay pass's FRI challenges and query plan (kept for the proof file)
    std::vector<F> fri_r;
    std::vector<int> which;
    std::vector<long> pos;
    // replay: the commitment's stream, synchronised only when the replay
    // reaches the commitment (the GKR part overlaps its tail), and the time
    // spent waiting for it
    vg_ctx *commit_ctx = nullptr;
    double commit_wait_s = 0;
};

struct vg_session {
    std::shared_ptr<CircuitData> circuit;
    vg_ctx *ctx = nullptr;
    vg_pc *pc = nullptr;
    zk_prover *p = nullptr;
    vg_ctx *cctx = nullptr;   // the commitment's context: its own stream, so the
                              // commitment overlaps the sumcheck rounds
    void *pub = nullptr;   // device buffer for the public eq table
    size_t pub_bytes = 0;
    bool loaded = false;   // false after a failed load: no valid circuit
    // input values set by vg_session_set_inputs (device; null: the circuit's own)
    void *inputs = nullptr, *inputs_raw = nullptr;
    size_t inputs_bytes = 0, inputs_raw_bytes = 0;
    bool inputs_on = false;
    // the fft_gkr side proof of every proof (on its own stream), made on first use
    vg_ctx *fctx = nullptr;
    vg_fft_gkr *fft = nullptr;
    int fft_max_lg = 0;
    bool fft_on = true;
    // the last proof, for vg_session_write_proof: the device results stay in
    // the objects' pinned buffers until the next proof
    bool last_valid = false;
    unsigned last_seed = 0;
    int last_proof_size = 0;
    PassResults last;
};

// The verifier runs `./fft_gkr <L - 6>` next to every proof of input size
// 2^L and counts its prover time (vpd_verifier.cpp:89-99); its random stream
// is that of a fresh process (seed 1).  Here it is launched on the session's
// third stream right after the proof's launch pass, so it runs beside the
// proof.  Returns the size launched, 0 when none (off, or L <= 6).
static int fft_side_launch(vg_session *s, int *lg_out)
{
    *lg_out = 0;
    const int lg = s->circuit->C.circuit[0].bit_length - 6;
    if (!s->fft_on || lg < 1) return VG_OK;
    int rc = VG_OK;
    if (!s->fctx) {
        int dev = 0;
        vg_ctx_device(s->ctx, &dev);
        rc = vg_ctx_create(dev, &s->fctx);
        if (rc != VG_OK) return rc;
    }
    if (!s->fft) {
        rc = vg_fft_gkr_create(s->fctx, lg, &s->fft);
        if (rc != VG_OK) return rc;
        s->fft_max_lg = lg;
    } else if (s->fft_max_lg < lg) {   // grown in place: no device-wide synchronisation
        rc = vg_fft_gkr_reserve(s->fft, lg);
        if (rc != VG_OK) return rc;
        s->fft_max_lg = lg;
    }
    rc = vg_fft_gkr_launch(s->fft, lg, 1);
    if (rc != VG_OK) {
        vg_ctx_sync(s->fctx);
        return rc;
    }
    *lg_out = lg;
    return VG_OK;
}

// Back to the circuit's own input values (a new circuit was loaded).
static void drop_inputs(vg_session *s)
{
    if (s->inputs_on && s->p && s->p->dev_gkr) vg_gkr_set_input(s->p->dev_gkr, nullptr);
    s->inputs_on = false;
}

extern "C" int vg_session_set_inputs(vg_session *s, const int64_t *values, long n)
{
    if (!s || !s->p || !values) return vg_fail(VG_ERR_ARG, "vg_session_set_inputs: null argument");
    if (!s->loaded) return vg_fail(VG_ERR_STATE, "vg_session_set_inputs: no circuit loaded");
    const long width = 1L << s->circuit->C.circuit[0].bit_length;
    if (n < 1 || n > width) return vg_fail(VG_ERR_ARG, "vg_session_set_inputs: %ld values for an input layer of %ld", n, width);
    int dev = 0;
    vg_ctx_device(s->ctx, &dev);
    cudaSetDevice(dev);
    int rc = vg_ctx_grow_dev(s->ctx, &s->inputs_raw, &s->inputs_raw_bytes, (size_t)n * 8);
    if (rc == VG_OK) rc = vg_ctx_grow_dev(s->ctx, &s->inputs, &s->inputs_bytes, (size_t)width * sizeof(F));
    if (rc == VG_OK) rc = vg_h2d_staged(s->ctx, s->inputs_raw, values, (size_t)n * 8);
    if (rc == VG_OK) rc = vg_input_values(s->ctx, (const int64_t *)s->inputs_raw, n, width, (vg_fe *)s->inputs);
    if (rc == VG_OK) rc = vg_gkr_set_input(s->p->dev_gkr, (const vg_fe *)s->inputs);
    // the commitment's stream reads the input layer too
    if (rc == VG_OK) rc = vg_ctx_wait_for(s->cctx, s->ctx);
    if (rc != VG_OK) {
        drop_inputs(s);
        return rc;
    }
    s->inputs_on = true;
    return VG_OK;
}

extern "C" int vg_session_set_fft_gkr(vg_session *s, int on)
{
    if (!s) return vg_fail(VG_ERR_ARG, "vg_session_set_fft_gkr: null session");
    s->fft_on = on != 0;
    return VG_OK;
}

// The sumcheck stream carries a proof's critical path (the layers' chain of
// phases); the commitment and the side proof run beside it on their own
// streams with room to spare.  So the sumcheck stream gets the device's
// highest priority and the others fill the SMs it leaves idle
// (VIRGO_STREAM_PRIORITY=0: all streams at the default priority).
static bool prioritise_sumcheck()
{
    const char *e = getenv("VIRGO_STREAM_PRIORITY");
    return !(e && e[0] == '0');
}

static int session_device(vg_ctx **ctx)
{
    int dev = 0;
    if (const char *e = getenv("VIRGO_DEVICE")) dev = atoi(e);
    int rc = vg_ctx_create(dev, ctx);
    if (rc == VG_OK && prioritise_sumcheck()) rc = vg_ctx_raise_priority(*ctx);
    return rc;
}

// own context, commitment state and prover over a (possibly shared) circuit
static int session_attach(vg_session *s)
{
    int rc = s->ctx ? VG_OK : session_device(&s->ctx);
    if (rc != VG_OK) return rc;
    rc = vg_ctx_set_hash(s->ctx, virgo_hash_kind());
    if (rc == VG_OK && !s->cctx) {
        int dev = 0;
        vg_ctx_device(s->ctx, &dev);
        rc = vg_ctx_create(dev, &s->cctx);
    }
    if (rc == VG_OK) rc = vg_ctx_set_hash(s->cctx, virgo_hash_kind());
    if (rc == VG_OK && !s->pc) rc = vg_pc_create(s->cctx, &s->pc);
    if (rc != VG_OK) return rc;
    if (!s->p) {
        s->p = new zk_prover();
        s->p->quiet = true;
    }
    s->p->attach_circuit(s->circuit->C, s->circuit->dev, s->ctx);
    return VG_OK;
}

static bool same_shape(const layered_circuit &a, const int *bl, int depth)
{
    if (!a.circuit || a.total_depth != depth) return false;
    for (int i = 0; i < depth; ++i)
        if (a.circuit[i].bit_length != bl[i]) return false;
    return true;
}

// Builds (or rebuilds in place) the session's device circuit from file-level
// layers; the reader's padding and relay layer are applied on the device.
extern "C" int vg_session_load(vg_session *s, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                               const void *const *v, int index_bytes)
{
    if (!s || !s->ctx || d < 1 || !n || !ty || !u || !v) return vg_fail(VG_ERR_ARG, "vg_session_load: bad argument");
    s->last_valid = false;
    int dev = 0;
    vg_ctx_device(s->ctx, &dev);
    cudaSetDevice(dev);
    if (!s->circuit || s->circuit.use_count() > 1) s->circuit = std::make_shared<CircuitData>();
    CircuitData *cd = s->circuit.get();
    std::vector<int> bl(d + 1);
    drop_inputs(s);
    s->loaded = false;
    int rc = vg_circuit_build(s->ctx, d, n, ty, u, v, index_bytes, &cd->dev, bl.data());
    if (rc != VG_OK) return rc;
    const bool keep = s->p && s->p->dev_circuit == cd->dev && same_shape(cd->C, bl.data(), d + 1);
    if (!same_shape(cd->C, bl.data(), d + 1)) {
        delete[] cd->C.circuit;
        cd->C.circuit = new layer[d + 1];
        cd->C.total_depth = d + 1;
        for (int i = 0; i <= d; ++i) cd->C.circuit[i].bit_length = bl[i];
    }
    if (keep) {
        s->p->C = cd->C;   // same widths: the prover's device tables still fit
        s->loaded = true;
        return VG_OK;
    }
    rc = session_attach(s);
    s->loaded = rc == VG_OK;
    return rc;
}

extern "C" int vg_session_new(vg_session **out)
{
    if (!out) return vg_fail(VG_ERR_ARG, "vg_session_new: null out");
    vg_session *s = new vg_session();
    int rc = session_device(&s->ctx);
    if (rc != VG_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return VG_OK;
}

extern "C" int vg_session_create(int d, const long *n, const uint8_t *const *ty, const int64_t *const *u,
                                 const int64_t *const *v, vg_session **out)
{
    if (!n || !ty || !u || !v || !out) return vg_fail(VG_ERR_ARG, "vg_session_create: bad argument");
    vg_session *s = new vg_session();
    int rc = session_device(&s->ctx);
    if (rc == VG_OK) rc = vg_session_load(s, d, n, ty, (const void *const *)u, (const void *const *)v, 8);
    if (rc != VG_OK) {
        vg_session_destroy(s);
        return rc;
    }
    *out = s;
    return VG_OK;
}

extern "C" int vg_session_fork(vg_session *base, vg_session **out)
{
    if (!base || !out) return vg_fail(VG_ERR_ARG, "vg_session_fork: null argument");
    if (!base->loaded) return vg_fail(VG_ERR_STATE, "vg_session_fork: the base session holds no circuit");
    vg_session *s = new vg_session();
    s->circuit = base->circuit;
    s->fft_on = base->fft_on;
    int rc = session_attach(s);
    s->loaded = rc == VG_OK;
    if (rc != VG_OK) {
        vg_session_destroy(s);
        return rc;
    }
    *out = s;
    return VG_OK;
}

// text circuit format of src/linear_gkr/README.md (the meta file is only
// needed by the verifier's predicate evaluation and is not read here)
extern "C" int vg_circuit_is_binary(const char *path);

extern "C" int vg_session_from_file(const char *circuit_path, vg_session **out)
{
    if (!circuit_path || !out) return vg_fail(VG_ERR_ARG, "vg_session_from_file: null argument");
    if (vg_circuit_is_binary(circuit_path)) {   // binary circuit file: mapped, no parsing
        vg_session *s = nullptr;
        int rc = vg_session_new(&s);
        if (rc == VG_OK) rc = vg_session_load_file(s, circuit_path);
        if (rc != VG_OK) {
            vg_session_destroy(s);
            return rc;
        }
        *out = s;
        return VG_OK;
    }
    FILE *f = fopen(circuit_path, "rb");
    if (!f) return vg_fail(VG_ERR_ARG, "cannot open circuit file");
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> buf(sz + 1);
    size_t got = fread(buf.data(), 1, sz, f);
    fclose(f);
    buf[got] = 0;
    const char *p = buf.data();
    auto next = [&](long long &x) -> bool {
        while (*p && (*p < '0' || *p > '9') && *p != '-') ++p;
        if (!*p) return false;
        bool neg = false;
        if (*p == '-') {
            neg = true;
            ++p;
        }
        long long r = 0;
        while (*p >= '0' && *p <= '9') r = r * 10 + (*p++ - '0');
        x = neg ? -r : r;
        return true;
    };
    long long d;
    if (!next(d) || d < 1 || d > 100000) return vg_fail(VG_ERR_ARG, "circuit file: bad depth");
    std::vector<long> n(d);
    std::vector<std::vector<uint8_t> > ty(d);
    std::vector<std::vector<int64_t> > u(d), v(d);
    for (long long i = 0; i < d; ++i) {
        long long cnt;
        if (!next(cnt) || cnt < 1) return vg_fail(VG_ERR_ARG, "circuit file: bad gate count");
        n[i] = (long)cnt;
        ty[i].resize(cnt);
        u[i].resize(cnt);
        v[i].resize(cnt);
        for (long long j = 0; j < cnt; ++j) {
            long long t, g, a, b;
            if (!next(t) || !next(g) || !next(a) || !next(b)) return vg_fail(VG_ERR_ARG, "circuit file: truncated gate");
            if (g != j) {
                fprintf(stderr, "Error, gates must be in sorted order, and full [0, 2^n - 1]. %lld %lld %lld\n", i + 1, j, g);
                return vg_fail(VG_ERR_ARG, "circuit file: bad gate");
            }
            ty[i][j] = (uint8_t)t;
            u[i][j] = a;
            v[i][j] = b;
        }
    }
    std::vector<const uint8_t *> pty(d);
    std::vector<const int64_t *> pu(d), pv(d);
    for (long long i = 0; i < d; ++i) {
        pty[i] = ty[i].data();
        pu[i] = u[i].data();
        pv[i] = v[i].data();
    }
    return vg_session_create((int)d, n.data(), pty.data(), pu.data(), pv.data(), out);
}

extern "C" int vg_session_destroy(vg_session *s)
{
    if (!s) return VG_OK;
    if (s->p) {
        s->p->delete_self();
        delete s->p;
    }
    if (s->pub) vg_dev_free(s->cctx, s->pub);
    if (s->ctx) {
        vg_ctx_sync(s->ctx);
        if (s->inputs) vg_dev_free(s->ctx, s->inputs);
        if (s->inputs_raw) vg_dev_free(s->ctx, s->inputs_raw);
    }
    if (s->fft) vg_fft_gkr_destroy(s->fft);
    if (s->fctx) vg_ctx_destroy(s->fctx);
    if (s->pc) vg_pc_destroy(s->pc);
    if (s->cctx) vg_ctx_destroy(s->cctx);
    s->circuit.reset();
    if (s->ctx) vg_ctx_destroy(s->ctx);
    delete s;
    return VG_OK;
}

extern "C" int vg_session_depth(vg_session *s, int *depth, int *input_log)
{
    if (!s) return vg_fail(VG_ERR_ARG, "vg_session_depth: null session");
    if (depth) *depth = s->circuit->C.total_depth;
    if (input_log) *input_log = s->circuit->C.circuit[0].bit_length;
    return VG_OK;
}

extern "C" void vg_free(void *p) { free(p); }

extern "C" int vg_session_commit_ctx(vg_session *s, vg_ctx **out)
{
    if (!s || !out) return vg_fail(VG_ERR_ARG, "vg_session_commit_ctx: null argument");
    *out = s->cctx;
    return VG_OK;
}

extern "C" int vg_session_ctx(vg_session *s, vg_ctx **out)
{
    if (!s || !out) return vg_fail(VG_ERR_ARG, "null argument");
    *out = s->ctx;
    return VG_OK;
}

extern "C" int vg_default_ctx(vg_ctx **out)
{
    if (!out) return vg_fail(VG_ERR_ARG, "null argument");
    *out = virgo::ctx();
    return VG_OK;
}

// decimal digits of x into p (x >= 0 or negative), returns the end
static char *put_int(char *p, long long x)
{
    char tmp[24];
    int n = 0;
    unsigned long long ux = x < 0 ? 0ULL - (unsigned long long)x : (unsigned long long)x;
    do {
        tmp[n++] = (char)('0' + ux % 10);
        ux /= 10;
    } while (ux);
    if (x < 0) *p++ = '-';
    while (n) *p++ = tmp[--n];
    return p;
}

extern "C" int vg_circuit_write_text(int d, const long *n, const uint8_t *const *ty, const int64_t *const *u,
                                     const int64_t *const *v, const char *circuit_path, const char *meta_path)
{
    if (d < 1 || !n || !ty || !u || !v || !circuit_path) return vg_fail(VG_ERR_ARG, "vg_circuit_write_text: bad argument");
    FILE *f = fopen(circuit_path, "wb");
    if (!f) return vg_fail(VG_ERR_ARG, "vg_circuit_write_text: cannot open output");
    std::vector<char> buf(1 << 22);
    char *p = buf.data();
    char *end = buf.data() + buf.size() - 128;
    auto flush = [&]() {
        fwrite(buf.data(), 1, p - buf.data(), f);
        p = buf.data();
    };
    p = put_int(p, d);
    *p++ = '\n';
    for (int i = 0; i < d; ++i) {
        p = put_int(p, n[i]);
        *p++ = ' ';
        for (long g = 0; g < n[i]; ++g) {
            if (p > end) flush();
            p = put_int(p, ty[i][g]);
            *p++ = ' ';
            p = put_int(p, g);
            *p++ = ' ';
            p = put_int(p, u[i][g]);
            *p++ = ' ';
            p = put_int(p, v[i][g]);
            if (g + 1 < n[i]) *p++ = ' ';
        }
        *p++ = '\n';
    }
    flush();
    fclose(f);
    if (meta_path) {
        FILE *m = fopen(meta_path, "wb");
        if (!m) return vg_fail(VG_ERR_ARG, "out of host memory");
        for (int i = 0; i < d; ++i) fputs("0 0 1 0 0\n", m);
        fclose(m);
    }
    return VG_OK;
}

// Open-addressing set of 64-bit keys (linear probing, power-of-two table,
// grown at half load) for the proof-size bookkeeping of the query answers:
// a few thousand operations per proof, where node-based sets cost a
// millisecond.
class KeySet {
    std::vector<uint64_t> t_;
    size_t n_ = 0;
    static constexpr uint64_t EMPTY = ~0ull;
    size_t slot(uint64_t k) const
    {
        size_t i = (size_t)((k * 0x9E3779B97F4A7C15ull) >> 20) & (t_.size() - 1);
        while (t_[i] != EMPTY && t_[i] != k) i = (i + 1) & (t_.size() - 1);
        return i;
    }

public:
    KeySet() : t_(1024, EMPTY) {}
    bool count(uint64_t k) const { return t_[slot(k)] == k; }
    bool insert(uint64_t k)   // true when k was not there
    {
        size_t i = slot(k);
        if (t_[i] == k) return false;
        t_[i] = k;
        if (2 * ++n_ > t_.size()) {
            std::vector<uint64_t> old(t_.size() * 2, EMPTY);
            old.swap(t_);
            for (uint64_t x : old)
                if (x != EMPTY) t_[slot(x)] = x;
        }
        return true;
    }
};

// One run of the protocol from srand(seed).  launch: every device step is
// enqueued and nothing is read back (the transcript is off); replay: no
// device work, every device result comes from `res`, and the transcript,
// the claim check and the proof-size bookkeeping are produced.  Both runs
// draw the same rand() values in the same order.
static int prove_pass(vg_session *s, unsigned seed, bool launch, PassResults &res, Transcript &tr, int &proof_size_out)
{
    struct random_data rd;
    int32_t statebuf[32];   // 128 bytes: glibc's default TYPE_3 state, as srand() uses
    memset(&rd, 0, sizeof rd);
    memset(statebuf, 0, sizeof statebuf);
    initstate_r(seed, (char *)statebuf, sizeof statebuf, &rd);
    prime_field::set_thread_random_state(&rd);
    struct Restore {
        ~Restore() { prime_field::set_thread_random_state(nullptr); }
    } restore;
    auto rand_int = [&]() {
        int32_t r;
        random_r(&rd, &r);
        return (int)r;
    };
    zk_prover &p = *s->p;
    layered_circuit &C = s->circuit->C;
    p.reset_proof();
    p.defer_mode = launch ? zk_prover::DEFER_LAUNCH : zk_prover::DEFER_REPLAY;
    p.replay = res.rec;
    p.replay_n = res.nrec;
    p.replay_i = 0;
    int proof_size = 0;

    // ---------------- GKR (zk_verifier.cpp:919-1207) ----------------
    F *result = p.evaluate();
    F alpha(1), beta(0);
    const int out_bl = C.circuit[C.total_depth - 1].bit_length;
    std::vector<F> r_0 = draws(out_bl), r_1 = draws(out_bl);
    std::vector<F> omr_0(out_bl), omr_1(out_bl);
    for (int i = 0; i < out_bl; ++i) {
        omr_0[i] = F(1) - r_0[i];
        omr_1[i] = F(1) - r_1[i];
    }
    F a_0 = p.V_res(omr_0.data(), r_0.data(), result, out_bl, 1 << out_bl);
    tr.fe('R', a_0);
    F alpha_beta_sum = alpha * a_0;
    std::vector<F> all_pub_mask;
    F all_mask_sum(0);

    for (int i = C.total_depth - 1; i >= 1; --i) {
        const int ll = C.circuit[i - 1].bit_length;
        F rho = prime_field::random();
        p.sumcheck_init(i, C.circuit[i].bit_length, ll, ll, alpha, beta, r_0.data(), r_1.data(), omr_0.data(), omr_1.data());
        p.generate_maskpoly_pre_rho(ll * 2 + 1, 2);
        p.rho = rho;
        p.generate_maskpoly_after_rho(ll * 2 + 1, 2);
        tr.fe('S', p.maskpoly_sumc);
        alpha_beta_sum = alpha_beta_sum + p.maskpoly_sumc;
        p.sumcheck_phase1_init();
        F previous_random(0);
        std::vector<F> r_u = draws(ll), r_v = draws(ll);
        F direct_relay_value = alpha * direct_relay(C, i, r_0.data(), r_u.data()) + beta * direct_relay(C, i, r_1.data(), r_u.data());
        F r_c = prime_field::random();
        if (i == 1) {
            for (int j = 0; j < ll; ++j) r_v[j] = F(0);
            r_c = F(0);
        }
        F random_combine = prime_field::random();
        F linear_coeff = prime_field::random();
        // public coefficients of the R mask at preu1 / prev1 (zk_verifier.cpp:983-990)
        const F pu1 = p.prepreu1, pv1 = p.preprev1, one(1);
        all_pub_mask.push_back(one * random_combine + linear_coeff * one * random_combine);
        all_pub_mask.push_back(pu1 * random_combine + linear_coeff * pv1 * random_combine);
        all_pub_mask.push_back(pu1 * pu1 * random_combine + linear_coeff * pv1 * pv1 * random_combine);
        all_pub_mask.push_back(r_c * random_combine + linear_coeff * r_c * random_combine);
        all_pub_mask.push_back(r_c * r_c * random_combine + linear_coeff * r_c * r_c * random_combine);
        all_pub_mask.push_back(pu1 * r_c * random_combine + linear_coeff * pv1 * r_c * random_combine);
        // public coefficients of the sumcheck mask polynomial (zk_verifier.cpp:1002-1025)
        F linear_combine = prime_field::random();
        for (int k = 0; k < ll; ++k) {
            all_pub_mask.push_back(linear_combine * r_u[k] * r_u[k] * rho);
            all_pub_mask.push_back(linear_combine * r_u[k] * rho);
        }
        for (int k = 0; k < ll; ++k) {
            all_pub_mask.push_back(linear_combine * r_v[k] * r_v[k] * rho);
            all_pub_mask.push_back(linear_combine * r_v[k] * rho);
        }
        all_pub_mask.push_back(linear_combine * r_c * r_c * rho);
        all_pub_mask.push_back(linear_combine * r_c * rho);
        all_pub_mask.push_back(linear_combine * one * rho);
        const F ul = r_u[ll - 1], vl = r_v[ll - 1];
        all_pub_mask.push_back(linear_combine * ul * ul * ul * ul * ul * rho);
        all_pub_mask.push_back(linear_combine * ul * ul * ul * ul * rho);
        all_pub_mask.push_back(linear_combine * ul * ul * ul * rho);
        all_pub_mask.push_back(linear_combine * vl * vl * vl * vl * vl * rho);
        all_pub_mask.push_back(linear_combine * vl * vl * vl * vl * rho);
        all_pub_mask.push_back(linear_combine * vl * vl * vl * rho);
        std::vector<F> omr_u(ll), omr_v(ll);
        for (int j = 0; j < ll; ++j) {
            omr_u[j] = F(1) - r_u[j];
            omr_v[j] = F(1) - r_v[j];
        }
        // phase 1
        for (int j = 0; j < ll; ++j) {
            if (j == ll - 1) {
                quintuple_poly poly = p.sumcheck_phase1_updatelastbit(previous_random, j);
                proof_size += sizeof(quintuple_poly);
                F u6[6] = {poly.a, poly.b, poly.c, poly.d, poly.e, poly.f};
                tr.put('p', u6, 6);
                alpha_beta_sum = poly.eval(r_u[j]);
            } else {
                quadratic_poly poly = p.sumcheck_phase1_update(previous_random, j);
                proof_size += sizeof(quadratic_poly);
                F u3[3] = {poly.a, poly.b, poly.c};
                tr.put('q', u3, 3);
                alpha_beta_sum = poly.eval(r_u[j]);
            }
            previous_random = r_u[j];
        }
        p.sumcheck_phase2_init(previous_random, r_u.data(), omr_u.data());
        tr.fe('u', p.v_u);
        previous_random = F(0);
        for (int j = 0; j < ll; ++j) {
            if (i == 1) r_v[j] = F(0);
            if (j == ll - 1) {
                quintuple_poly poly = p.sumcheck_phase2_updatelastbit(previous_random, j);
                proof_size += sizeof(quintuple_poly);
                F u6[6] = {poly.a, poly.b, poly.c, poly.d, poly.e, poly.f};
                tr.put('P', u6, 6);
                alpha_beta_sum = poly.eval(r_v[j]) + direct_relay_value * p.v_u;
            } else {
                quadratic_poly poly = p.sumcheck_phase2_update(previous_random, j);
                proof_size += sizeof(quadratic_poly);
                F u3[3] = {poly.a, poly.b, poly.c};
                tr.put('Q', u3, 3);
                alpha_beta_sum = poly.eval(r_v[j]) + direct_relay_value * p.v_u;
            }
            previous_random = r_v[j];
        }
        auto claims = p.sumcheck_finalize(previous_random);
        F cl[2] = {claims.first, claims.second};
        tr.put('z', cl, 2);
        const F v_u = claims.first;
        // final round with the general value implied by the claim
        quadratic_poly fin = p.sumcheck_finalround(previous_random, ll << 1, F(0));
        F general = alpha_beta_sum - direct_relay_value * v_u - (fin.a + fin.b + fin.c + fin.c);
        fin.b = fin.b + general;
        F u3[3] = {fin.a, fin.b, fin.c};
        tr.put('f', u3, 3);
        if (i == 1) r_c = F(0);
        alpha_beta_sum = fin.eval(r_c) + direct_relay_value * p.v_u;
        F mv = p.query(r_u.data(), r_v.data(), r_c);
        tr.fe('y', mv);
        F g1 = p.queryRg1(r_c);
        tr.fe('g', g1);
        F g2 = p.queryRg2(r_c);
        tr.fe('h', g2);
        all_mask_sum = all_mask_sum + g1 * random_combine + linear_coeff * g2 * random_combine + linear_combine * mv;
        alpha = prime_field::random();
        beta = prime_field::random();
        alpha_beta_sum = i != 1 ? alpha * v_u + beta * claims.second : v_u;
        r_0 = r_u;
        r_1 = r_v;
        omr_0 = omr_u;
        omr_1 = omr_v;
    }
    all_pub_mask.push_back(p.Zu);
    all_pub_mask.push_back(p.Zu * p.preu1);
    p.all_pri_mask.push_back(p.maskr[0]);
    p.all_pri_mask.push_back(p.maskr[1]);
    all_mask_sum = all_mask_sum + p.Zu * p.sumRc.eval(p.preu1);

    // ---------------- commitments (zk_verifier.cpp:1210-1219; poly_commit.h:42-351) ----------------
    const int L = C.circuit[0].bit_length;
    const long M = vg_pc_mask_len(L, (long)p.all_pri_mask.size());
    if ((long)all_pub_mask.size() > M) return vg_fail(VG_ERR_STATE, "vg_session_prove: public mask longer than the slice");
    while ((long)all_pub_mask.size() < M) all_pub_mask.push_back(F(0));   // poly_commit.h:138-139

    // FRI challenges (vpd_verifier.cpp:46-78): one per fold
    std::vector<F> fri_r;
    for (int cw = 1 << (L + rs_code_rate - log_slice_number); cw > (1 << rs_code_rate); cw /= 2)
        fri_r.push_back(prime_field::random());
    const int levels = (int)fri_r.size();

    // query positions (vpd_verifier.cpp:105-312): from the rand() stream alone
    std::vector<int> which;
    std::vector<long> pos;
    for (int rep = 0; rep < ldt_repeat_num; ++rep) {
        long long pw = 0;
        for (int i = 0; i < L - log_slice_number; ++i) {
            const int lw = L + rs_code_rate - log_slice_number - i;
            if (i == 0) {
                do {
                    pw = rand_int() % (1 << lw);
                } while (pw < (1 << (L - log_slice_number - i)) || pw % 2 == 1);
                which.push_back(0);
                pos.push_back((long)(pw / 2));
                which.push_back(1);
                pos.push_back((long)(pw / 2));
            } else {
                pw = pw % (1 << lw);
            }
            which.push_back(2 + i);
            pos.push_back((long)(pw / 2));
        }
    }
    const int nq = (int)which.size();

    if (launch) {
        const size_t pub_bytes = ((size_t)1 << L) * sizeof(F);
        if (s->pub_bytes < pub_bytes) {   // stream ordered on the commitment stream: no device-wide wait
            int rc = vg_ctx_grow_dev(s->cctx, &s->pub, &s->pub_bytes, pub_bytes);
            if (rc != VG_OK) return rc;
        }
        // the commitment depends on no GKR device result: it runs on its own
        // stream, concurrently with the sumcheck work enqueued above
        int rc = vg_eq_table_async(s->cctx, (const vg_fe *)r_0.data(), L, (vg_fe *)s->pub);
        if (rc == VG_OK)
            rc = vg_pc_prove_deferred(s->pc, (const vg_fe *)p.circuit_value[0], L, (const vg_fe *)p.all_pri_mask.data(),
                                      (long)p.all_pri_mask.size(), (const vg_fe *)s->pub,
                                      (const vg_fe *)all_pub_mask.data(), M, (const vg_fe *)fri_r.data(), levels, nq,
                                      which.data(), pos.data(), &res.pc);
        res.levels = levels;
        return rc;
    }

    // ---- replay: commitment messages ----
    if (res.commit_ctx) {
        const auto w0 = std::chrono::steady_clock::now();
        const int rc = vg_ctx_sync(res.commit_ctx);
        res.commit_wait_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
        if (rc != VG_OK) return rc;
    }
    const vg_pc_results &pr = res.pc;
    res.fri_r = fri_r;
    res.which = which;
    res.pos = pos;
    // the claimed inner product the reference asserts (poly_commit.h:193)
    const F target = alpha_beta_sum - p.Zu * p.sumRc.eval(p.preu1) + all_mask_sum;
    const F inner = *(const F *)pr.inner;
    if (inner != target)
        return vg_fail(VG_ERR_STATE, "vg_session_prove: committed inner product differs from the sumcheck claim");
    const __hhash_digest *roots = (const __hhash_digest *)pr.roots;
    tr.put('C', &roots[0], 2);
    tr.put('C', &roots[1], 2);
    proof_size += 2 * sizeof(__hhash_digest);
    tr.put('A', pr.all_sum, slice_number + 1);
    tr.put('B', roots, 4);
    for (int t = 0; t < levels; ++t) tr.put('T', &roots[2 + t], 2);
    {
        // the final level in the interleaved layout of fri.cpp:348-363 and 382-388
        const long n = pr.n_final, h = n >> 1;
        const F *b = (const F *)pr.final_cw;
        std::vector<F> data((size_t)n * slice_number), msk(n);
        for (long j = 0; j < h; ++j) {
            for (int sl = 0; sl < slice_number; ++sl) {
                data[(j << 7) | (sl << 1) | 0] = b[sl * n + j];
                data[(j << 7) | (sl << 1) | 1] = b[sl * n + j + h];
            }
            msk[2 * j] = b[64 * n + j];
            msk[2 * j + 1] = b[64 * n + j + h];
        }
        tr.put('X', data.data(), (uint32_t)(n * slice_number));
        tr.put('x', msk.data(), (uint32_t)n);
    }

    // ---- replay: query answers and the proof-size bookkeeping (fri.cpp:148-289) ----
    const F *qvals = (const F *)pr.qvals;
    const __hhash_digest *qpaths = (const __hhash_digest *)pr.qpaths;
    KeySet seen_elem[2], seen_node[2];
    std::vector<KeySet> seen_level(levels);
    const long long half_S = 1LL << (L - 2);
    for (int q = 0; q < nq; ++q) {
        std::pair<std::vector<std::pair<F, F> >, std::vector<__hhash_digest> > a;
        const F *v = &qvals[(size_t)q * 130];
        for (int k = 0; k <= slice_number; ++k) a.first.push_back(std::make_pair(v[2 * k], v[2 * k + 1]));
        const __hhash_digest *pth = &qpaths[(size_t)q * 32];
        const int depth = which[q] < 2 ? L - 2 : L - (which[q] - 2) - 3;   // log2 of the set's leaf count
        int new_size = 0;
        if (which[q] < 2) {   // fri::request_init_value_with_merkle
            const int o = which[q];
            const long long p0 = pos[q];
            // the reference marks the 2 x 64 elements of position p0 together
            // (fri.cpp:166-176), so they are new exactly when p0 is
            if (seen_elem[o].insert((uint64_t)p0)) new_size += 2 * slice_number * (int)sizeof(F);
            a.second.resize(depth + 1);
            a.second[depth] = pth[depth];
            long long node = p0 + half_S;
            for (int k = 0; k < depth; ++k) {
                if (!seen_node[o].count((uint64_t)(node ^ 1))) new_size += sizeof(__hhash_digest);
                seen_node[o].insert((uint64_t)node);
                seen_node[o].insert((uint64_t)(node ^ 1));
                a.second[k] = pth[k];
                node /= 2;
            }
            tr.answer('I', a, new_size);
            if (o == 1) proof_size += new_size;   // the verifier adds the second call's count
        } else {              // fri::request_step_commit
            const int lvl = which[q] - 2;
            const long long h = 1LL << depth, p0 = pos[q] % h;
            auto &seen = seen_level[lvl];
            // the reference tests element keys in the array that marks Merkle
            // nodes (fri.cpp:252-262); the keys 2^(lss+1) p0 + 2k can only
            // meet a node index below 2h
            bool visited = false;
            if ((p0 << (log_slice_number + 1)) < 2 * h)
                for (int k = 0; k < slice_number && !visited; ++k)
                    if (seen.count((uint64_t)((p0 << (log_slice_number + 1)) | (k << 1)))) visited = true;
            if (!visited) new_size += sizeof(F);
            long long node = p0 + h;
            int k = 0;
            while (node != 1) {
                if (!seen.count((uint64_t)(node ^ 1))) {
                    new_size += sizeof(__hhash_digest);
                    seen.insert((uint64_t)(node ^ 1));
                    seen.insert((uint64_t)node);
                }
                a.second.push_back(pth[k++]);
                node /= 2;
            }
            a.second.push_back(pth[depth]);
            tr.answer('J', a, new_size);
            proof_size += new_size;
        }
    }
    if (p.replay_i != res.nrec) return vg_fail(VG_ERR_STATE, "replay used %d of %d device records", p.replay_i, res.nrec);
    proof_size_out = proof_size;
    return VG_OK;
}

extern "C" int vg_session_prove(vg_session *s, unsigned seed, int want_transcript, vg_proof_stats *stats,
                                uint8_t **transcript, size_t *transcript_len)
{
    if (!s || !s->p) return vg_fail(VG_ERR_ARG, "vg_session_prove: null session");
    if (!s->loaded) return vg_fail(VG_ERR_STATE, "vg_session_prove: no circuit loaded (the last load failed)");
    {
        int dev = 0;
        vg_ctx_device(s->ctx, &dev);
        cudaSetDevice(dev);   // this thread may not have used the session's device yet
    }
    auto t_all = clk::now();
    vg_proof_stats st;
    memset(&st, 0, sizeof st);
    long long launches0 = 0;
    vg_ctx_launch_count(s->ctx, &launches0);
    for (vg_ctx *x : {s->cctx, s->fctx}) {
        long long l2 = 0;
        if (x) vg_ctx_launch_count(x, &l2);
        launches0 += l2;
    }
    s->last_valid = false;   // the objects' result buffers are about to be reused
    zk_prover &p = *s->p;
    long long greplay0 = 0, gcap0 = 0;
    vg_gkr_graph_counts(p.dev_gkr, &greplay0, &gcap0);

    // launch pass: the whole proof enqueued on the session's stream
    PassResults res;
    Transcript tr;
    tr.on = false;
    int proof_size = 0;
    int rc = vg_gkr_defer(p.dev_gkr, 1);
    if (rc == VG_OK) rc = prove_pass(s, seed, true, res, tr, proof_size);
    const vg_fe *recs = nullptr;
    if (rc == VG_OK) rc = vg_gkr_records(p.dev_gkr, &recs, &res.nrec);
    vg_gkr_defer(p.dev_gkr, 0);
    p.defer_mode = zk_prover::DEFER_OFF;
    if (rc != VG_OK) {
        vg_ctx_sync(s->ctx);   // drain what was enqueued before the error
        vg_ctx_sync(s->cctx);
        return rc;
    }
    st.launch_s = since(t_all);
    auto t0 = clk::now();
    int fft_lg = 0;
    const int rc_fft = fft_side_launch(s, &fft_lg);   // host work hidden behind the proof's device time
    // the side proof's own stream is waited for after the replay, which also
    // overlaps its tail
    auto finish_side = [&](bool check) -> int {
        if (!fft_lg) return VG_OK;
        vg_fft_gkr_stats fs;
        const int r = vg_fft_gkr_finish(s->fft, &fs, nullptr, nullptr);
        fft_lg = check ? fft_lg : 0;
        if (!check || r != VG_OK) return r;
        if (!fs.pass) return vg_fail(VG_ERR_STATE, "fft_gkr side proof (lg %d) failed its checks", fft_lg);
        st.fft_gkr_s = fs.gpu_s;
        st.fft_gkr_lg = fft_lg;
        st.fft_gkr_proof_size = fs.proof_size;
        return VG_OK;
    };
    // the GKR records are on the host once the sumcheck stream is done; the
    // replay's commitment part waits for the commitment stream itself
    rc = vg_ctx_sync(s->ctx);
    if (rc == VG_OK) rc = rc_fft;
    if (rc != VG_OK) {
        vg_ctx_sync(s->cctx);
        finish_side(false);   // wait for the side proof and clear its run
        return rc;
    }
    st.wait_s = since(t0);

    // replay pass: messages, checks and the transcript from the device results
    t0 = clk::now();
    res.rec = (const F *)recs;
    res.commit_ctx = s->cctx;
    res.commit_wait_s = 0;
    tr.on = want_transcript != 0;
    rc = prove_pass(s, seed, false, res, tr, proof_size);
    p.defer_mode = zk_prover::DEFER_OFF;
    p.replay = nullptr;
    if (rc != VG_OK) {
        vg_ctx_sync(s->cctx);
        finish_side(false);
        return rc;
    }
    const auto t1 = clk::now();
    rc = finish_side(true);
    if (rc != VG_OK) return rc;
    const double side_wait = std::chrono::duration<double>(clk::now() - t1).count();
    st.replay_s = since(t0) - res.commit_wait_s - side_wait;
    st.wait_s += res.commit_wait_s + side_wait;
    st.prove_time = st.launch_s + st.wait_s;
    s->last = std::move(res);
    s->last_seed = seed;
    s->last_proof_size = proof_size;
    s->last_valid = true;

    st.total_s = since(t_all);
    st.proof_size = proof_size;
    long long launches1 = 0;
    vg_ctx_launch_count(s->ctx, &launches1);
    for (vg_ctx *x : {s->cctx, s->fctx}) {
        long long l2 = 0;
        if (x) vg_ctx_launch_count(x, &l2);
        launches1 += l2;
    }
    st.launches = launches1 - launches0;
    {
        long long gr = 0, gc = 0;
        vg_gkr_graph_counts(p.dev_gkr, &gr, &gc);
        st.graph_replays = (int)(gr - greplay0);
        st.graph_captures = (int)(gc - gcap0);
    }
    if (stats) *stats = st;
    if (transcript && transcript_len) {
        *transcript_len = tr.bytes.size();
        *transcript = (uint8_t *)malloc(tr.bytes.size() ? tr.bytes.size() : 1);
        if (tr.bytes.size()) memcpy(*transcript, tr.bytes.data(), tr.bytes.size());
    }
    return VG_OK;
}

// The last proof as a file (format in include/virgo_b200.h): every device
// result the prover's replay consumes, so a process with the circuit and the
// seed can answer the reference verifier's calls without a GPU.
extern "C" int vg_session_write_proof(vg_session *s, const char *path)
{
    if (!s || !path) return vg_fail(VG_ERR_ARG, "vg_session_write_proof: null argument");
    if (!s->last_valid) return vg_fail(VG_ERR_STATE, "vg_session_write_proof: no proof since the last load");
    const PassResults &r = s->last;
    const layered_circuit &C = s->circuit->C;
    const int depth = C.total_depth, levels = r.levels, nq = (int)r.which.size();
    const int64_t n_final = r.pc.n_final;
    if ((int)r.fri_r.size() != levels || (int)r.pos.size() != nq)
        return vg_fail(VG_ERR_STATE, "vg_session_write_proof: inconsistent proof state");
    FILE *f = fopen(path, "wb");
    if (!f) return vg_fail(VG_ERR_ARG, "vg_session_write_proof: cannot open %s", path);
    bool ok = true;
    auto put = [&](const void *p, size_t n) {
        if (ok && n && fwrite(p, 1, n, f) != n) ok = false;
    };
    const uint32_t version = 1, seed = s->last_seed;
    put("VGPF", 4);
    put(&version, 4);
    put(&seed, 4);
    put(&depth, 4);
    for (int i = 0; i < depth; ++i) {
        const int32_t bl = C.circuit[i].bit_length;
        put(&bl, 4);
    }
    const int32_t nrec = r.nrec, psize = s->last_proof_size;
    put(&nrec, 4);
    put(&levels, 4);
    put(&nq, 4);
    put(&n_final, 8);
    put(&psize, 4);
    put(r.rec, (size_t)nrec * 9 * sizeof(F));
    put(r.pc.roots, (size_t)(2 + levels) * sizeof(vg_digest));
    put(r.pc.all_sum, (size_t)(slice_number + 1) * sizeof(vg_fe));
    put(r.pc.inner, sizeof(vg_fe));
    put(r.fri_r.data(), (size_t)levels * sizeof(F));
    put(r.pc.final_cw, (size_t)(slice_number + 1) * n_final * sizeof(vg_fe));
    for (int q = 0; q < nq; ++q) {
        const int32_t w = r.which[q];
        put(&w, 4);
    }
    for (int q = 0; q < nq; ++q) {
        const int64_t p = r.pos[q];
        put(&p, 8);
    }
    put(r.pc.qvals, (size_t)nq * 130 * sizeof(vg_fe));
    put(r.pc.qpaths, (size_t)nq * 32 * sizeof(vg_digest));
    if (fclose(f) != 0) ok = false;
    if (!ok) return vg_fail(VG_ERR_ARG, "vg_session_write_proof: writing %s failed", path);
    return VG_OK;
}

// Proofs of several sessions at once, one host thread per session; each
// session has its own CUDA stream, so their kernels overlap on the GPU.
extern "C" int vg_session_prove_batch(vg_session *const *ss, int n, const unsigned *seeds, int want_transcript,
                                      vg_proof_stats *stats, uint8_t **transcripts, size_t *transcript_lens)
{
    if (!ss || !seeds || n < 0) return vg_fail(VG_ERR_ARG, "vg_session_prove_batch: bad argument");
    std::vector<int> rcs(n, VG_OK);
    std::vector<std::string> msgs(n);   // the error text is per thread: carry it back
    std::vector<std::thread> th;
    for (int i = 0; i < n; ++i)
        th.emplace_back([&, i]() {
            rcs[i] = vg_session_prove(ss[i], seeds[i], want_transcript, stats ? &stats[i] : nullptr,
                                      transcripts ? &transcripts[i] : nullptr, transcript_lens ? &transcript_lens[i] : nullptr);
            if (rcs[i] != VG_OK) msgs[i] = vg_last_error();
        });
    for (auto &t : th) t.join();
    for (int i = 0; i < n; ++i)
        if (rcs[i] != VG_OK) return vg_fail(rcs[i], "session %d: %s", i, msgs[i].c_str());
    return VG_OK;
}
