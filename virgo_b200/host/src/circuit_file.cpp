// Binary circuit files: the layers in exactly the layout vg_session_load
// takes, so loading is a memory map and a device build, with no parsing.
// The reference reads a text file with fscanf (zk_verifier.cpp:15-217),
// seconds at 2^24 gates.
//
// Layout (little endian, every section starting on an 8-byte boundary):
//   char magic[4] = "VGC1"; uint32 version = 1; uint32 d; uint32 index_bytes
//   int64 n[d]                       gates per file layer, input layer first
//   per layer i: uint8 ty[n[i]]; then u[n[i]] and v[n[i]], each element
//   8 bytes for the input layer (its u are the input values) and
//   index_bytes (4 or 8) for the others.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <cstdio>
#include <cstring>
#include <vector>
#include "virgo_b200.h"

int vg_fail(int code, const char *fmt, ...);

namespace
{
const char MAGIC[4] = {'V', 'G', 'C', '1'};
inline size_t up8(size_t x) { return (x + 7) & ~(size_t)7; }

struct Header {
    char magic[4];
    uint32_t version, d, index_bytes;
};

// Offsets of every section; false if the sizes do not fit `size` bytes.
bool layout(const Header &h, const int64_t *n, size_t size, std::vector<size_t> &off)
{
    size_t p = up8(sizeof(Header) + (size_t)h.d * 8);
    off.assign(3 * (size_t)h.d, 0);
    for (uint32_t i = 0; i < h.d; ++i) {
        if (n[i] < 1 || n[i] > (1LL << 30)) return false;
        const size_t wb = i == 0 ? 8 : h.index_bytes;
        off[3 * i] = p;
        p = up8(p + (size_t)n[i]);
        off[3 * i + 1] = p;
        p = up8(p + (size_t)n[i] * wb);
        off[3 * i + 2] = p;
        p = up8(p + (size_t)n[i] * wb);
        if (p > size) return false;
    }
    return true;
}

struct Mapped {
    void *base = MAP_FAILED;
    size_t size = 0;
    ~Mapped()
    {
        if (base != MAP_FAILED) munmap(base, size);
    }
};

int map_file(const char *path, Mapped &m, const Header *&h, const int64_t *&n, std::vector<size_t> &off)
{
    int fd = open(path, O_RDONLY);
    if (fd < 0) return vg_fail(VG_ERR_ARG, "cannot open circuit file %s", path);
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < (off_t)sizeof(Header)) {
        close(fd);
        return vg_fail(VG_ERR_ARG, "%s: not a binary circuit file", path);
    }
    m.size = (size_t)st.st_size;
    m.base = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (m.base == MAP_FAILED) return vg_fail(VG_ERR_ARG, "%s: mmap failed", path);
    h = (const Header *)m.base;
    if (memcmp(h->magic, MAGIC, 4) || h->version != 1 || h->d < 1 || h->d > 100000 ||
        (h->index_bytes != 4 && h->index_bytes != 8) || sizeof(Header) + (size_t)h->d * 8 > m.size)
        return vg_fail(VG_ERR_ARG, "%s: bad binary circuit header", path);
    n = (const int64_t *)((const char *)m.base + sizeof(Header));
    if (!layout(*h, n, m.size, off)) return vg_fail(VG_ERR_ARG, "%s: truncated binary circuit", path);
    return VG_OK;
}
}  // namespace

extern "C" int vg_circuit_is_binary(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return 0;
    char m[4] = {0, 0, 0, 0};
    const size_t got = fread(m, 1, 4, f);
    fclose(f);
    return got == 4 && !memcmp(m, MAGIC, 4);
}

extern "C" int vg_circuit_write_binary(const char *path, int d, const long *n, const uint8_t *const *ty,
                                       const void *const *u, const void *const *v, int index_bytes)
{
    if (!path || d < 1 || !n || !ty || !u || !v || (index_bytes != 4 && index_bytes != 8))
        return vg_fail(VG_ERR_ARG, "vg_circuit_write_binary: bad argument");
    FILE *f = fopen(path, "wb");
    if (!f) return vg_fail(VG_ERR_ARG, "cannot create %s", path);
    Header h;
    memcpy(h.magic, MAGIC, 4);
    h.version = 1;
    h.d = (uint32_t)d;
    h.index_bytes = (uint32_t)index_bytes;
    std::vector<int64_t> nn(n, n + d);
    const char zeros[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t pos = 0;
    bool ok = fwrite(&h, sizeof h, 1, f) == 1 && fwrite(nn.data(), 8, d, f) == (size_t)d;
    pos = sizeof h + 8 * (size_t)d;
    auto put = [&](const void *p, size_t bytes) {
        ok = ok && (bytes == 0 || fwrite(p, 1, bytes, f) == bytes);
        pos += bytes;
        const size_t pad = up8(pos) - pos;
        ok = ok && (pad == 0 || fwrite(zeros, 1, pad, f) == pad);
        pos += pad;
    };
    put(nullptr, 0);   // align the first section
    for (int i = 0; i < d && ok; ++i) {
        if (n[i] < 1) ok = false;
        const size_t wb = i == 0 ? 8 : (size_t)index_bytes;
        put(ty[i], (size_t)n[i]);
        put(u[i], (size_t)n[i] * wb);
        put(v[i], (size_t)n[i] * wb);
    }
    if (fclose(f) != 0) ok = false;
    return ok ? VG_OK : vg_fail(VG_ERR_ARG, "writing %s failed", path);
}

extern "C" int vg_circuit_binary_info(const char *path, int *d, int *index_bytes, long *n, int n_cap)
{
    if (!path || !d) return vg_fail(VG_ERR_ARG, "vg_circuit_binary_info: null argument");
    Mapped m;
    const Header *h;
    const int64_t *nn;
    std::vector<size_t> off;
    int rc = map_file(path, m, h, nn, off);
    if (rc != VG_OK) return rc;
    *d = (int)h->d;
    if (index_bytes) *index_bytes = (int)h->index_bytes;
    if (n)
        for (int i = 0; i < (int)h->d && i < n_cap; ++i) n[i] = (long)nn[i];
    return VG_OK;
}

extern "C" int vg_session_load_file(vg_session *s, const char *path)
{
    if (!s || !path) return vg_fail(VG_ERR_ARG, "vg_session_load_file: null argument");
    Mapped m;
    const Header *h;
    const int64_t *nn;
    std::vector<size_t> off;
    int rc = map_file(path, m, h, nn, off);
    if (rc != VG_OK) return rc;
    const int d = (int)h->d;
    std::vector<long> n(nn, nn + d);
    std::vector<const uint8_t *> ty(d);
    std::vector<const void *> u(d), v(d);
    const char *b = (const char *)m.base;
    for (int i = 0; i < d; ++i) {
        ty[i] = (const uint8_t *)(b + off[3 * i]);
        u[i] = b + off[3 * i + 1];
        v[i] = b + off[3 * i + 2];
    }
    // the map stays until the load (which ends with a synchronisation) returns
    return vg_session_load(s, d, n.data(), ty.data(), u.data(), v.data(), (int)h->index_bytes);
}
