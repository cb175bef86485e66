// lmb_lmfile.cu -- the `.lm` trajectory writer (include/lmb_lmfile.h).
//
// The HDF5 structures are encoded here from the HDF5 File Format
// Specification in the forms libhdf5 writes with its default file-creation
// properties: superblock version 0 (symbol-table leaf K 4, group B-tree K 16,
// chunk B-tree K 32), version-1 object headers, groups as symbol tables
// (version-1 B-tree of type 0 over symbol-table nodes, names in a local
// heap), dataspace version 1, datatype version 1, fill value version 2,
// layout version 3 (contiguous, or chunked over a version-1 B-tree of type
// 1), filter pipeline version 1 (deflate), attribute version 1.  All
// addresses are relative to the superblock, which follows the 512-byte user
// block; the superblock's end-of-file field is absolute, as libhdf5 stores it.
//
// Bulk data (compressed frame chunks, model tables) is appended as it
// arrives.  A flush appends the whole metadata tree after it and rewrites the
// superblock to point at the new root, so the file is complete after every
// flush; metadata left behind by earlier flushes is unreferenced space.
#include "lmb_internal.h"
#include "lmb_lmfile.h"

#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/resource.h>
#include <sys/stat.h>
#include <sys/syscall.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr uint64_t UNDEF = ~0ull;
constexpr uint64_t USER_BLOCK = 512;     // SimulationFile_create.cpp: H5Pset_userblock(512)
constexpr uint64_t SUPERBLOCK = 96;      // version 0 with 8-byte offsets and lengths
constexpr uint32_t SYM_LEAF_K = 4;       // symbol-table node: up to 8 entries
constexpr uint32_t BTREE_K = 16;         // group B-tree node: up to 32 children
constexpr uint32_t ISTORE_K = 32;        // chunk B-tree node: up to 64 chunks
constexpr uint64_t FRAME_CHUNK = 16;     // TUNE_LATTICE_GZIP_CHUNK_SIZE (src/cmake/options.cmake:84)
constexpr int FRAME_GZIP = 1;            // TUNE_LATTICE_GZIP_COMPRESSION_LEVEL (options.cmake:85)
constexpr uint64_t ROW_CHUNK = 100;      // chunk rows of the extendable datasets (SimulationFile.cpp:2194)
constexpr uint32_t FORMAT_VERSION = 4;   // SimulationFile::CURRENT_VERSION (SimulationFile.cpp:77)
constexpr int PINNED_SLOTS = 3;          // device frames in flight to the writer thread

struct Bytes {
    std::vector<uint8_t> v;
    void le(uint64_t x, int n)
    {
        for (int i = 0; i < n; i++) v.push_back((uint8_t)(x >> (8 * i)));
    }
    void u8(uint64_t x) { le(x, 1); }
    void u16(uint64_t x) { le(x, 2); }
    void u32(uint64_t x) { le(x, 4); }
    void u64(uint64_t x) { le(x, 8); }
    void raw(const void *p, size_t n)
    {
        if (!n) return;
        const uint8_t *b = (const uint8_t *)p;
        v.insert(v.end(), b, b + n);
    }
    void raw(const Bytes &b) { v.insert(v.end(), b.v.begin(), b.v.end()); }
    void zeros(size_t n) { v.insert(v.end(), n, 0); }
    void pad8()
    {
        while (v.size() % 8) v.push_back(0);
    }
    size_t size() const { return v.size(); }
};

enum class Type { U8, I8, U16, I16, U32, I32, U64, I64, F32, F64, STR };

uint32_t type_size(Type t, uint32_t strsize)
{
    switch (t) {
    case Type::U8:
    case Type::I8: return 1;
    case Type::U16:
    case Type::I16: return 2;
    case Type::U32:
    case Type::I32:
    case Type::F32: return 4;
    case Type::U64:
    case Type::I64:
    case Type::F64: return 8;
    case Type::STR: return strsize;
    }
    return 0;
}

bool is_signed(Type t) { return t == Type::I8 || t == Type::I16 || t == Type::I32 || t == Type::I64; }

// Datatype message, version 1: little-endian fixed point (signed bit for
// I32), IEEE double, or a null-terminated ASCII string of fixed size.
Bytes datatype(Type t, uint32_t strsize = 0)
{
    Bytes b;
    switch (t) {
    case Type::U8:
    case Type::I8:
    case Type::U16:
    case Type::I16:
    case Type::U32:
    case Type::I32:
    case Type::U64:
    case Type::I64: {
        const uint32_t n = type_size(t, 0);
        b.u8(0x10);
        b.u8(is_signed(t) ? 0x08 : 0x00);
        b.u8(0);
        b.u8(0);
        b.u32(n);
        b.u16(0);
        b.u16(8 * n);
        break;
    }
    case Type::F32:
        b.u8(0x11);
        b.u8(0x20);
        b.u8(31);
        b.u8(0);
        b.u32(4);
        b.u16(0);
        b.u16(32);
        b.u8(23);
        b.u8(8);
        b.u8(0);
        b.u8(23);
        b.u32(127);
        break;
    case Type::F64:
        b.u8(0x11);
        b.u8(0x20);  // mantissa normalisation: implied leading bit
        b.u8(63);    // sign bit position
        b.u8(0);
        b.u32(8);
        b.u16(0);
        b.u16(64);
        b.u8(52);
        b.u8(11);
        b.u8(0);
        b.u8(52);
        b.u32(1023);
        break;
    case Type::STR:
        b.u8(0x13);
        b.u8(0x00);
        b.u8(0);
        b.u8(0);
        b.u32(strsize);
        break;
    }
    return b;
}

// Dataspace message, version 1; rank 0 is a scalar.  An extendable dataset
// has an unlimited first dimension.
Bytes dataspace(const std::vector<uint64_t> &dims, bool extendable)
{
    Bytes b;
    b.u8(1);
    b.u8(dims.size());
    b.u8(extendable ? 1 : 0);
    b.u8(0);
    b.u32(0);
    for (uint64_t d : dims) b.u64(d);
    if (extendable)
        for (size_t i = 0; i < dims.size(); i++) b.u64(i == 0 ? UNDEF : dims[i]);
    return b;
}

struct Attr {
    std::string name;
    Type type;
    uint32_t strsize;
    std::vector<uint64_t> dims;
    std::vector<uint8_t> data;
};

Bytes attribute(const Attr &a)
{
    const Bytes dt = datatype(a.type, a.strsize), ds = dataspace(a.dims, false);
    Bytes b;
    b.u8(1);
    b.u8(0);
    b.u16(a.name.size() + 1);
    b.u16(dt.size());
    b.u16(ds.size());
    b.raw(a.name.c_str(), a.name.size() + 1);
    b.pad8();
    b.raw(dt);
    b.pad8();
    b.raw(ds);
    b.pad8();
    b.raw(a.data.data(), a.data.size());
    b.pad8();
    return b;
}

struct Chunk {
    std::vector<uint64_t> offset;  // element offsets, rank entries
    uint64_t addr;
    uint32_t nbytes;
};

struct Node {
    bool group = true;
    std::map<std::string, std::unique_ptr<Node>> children;  // byte order = strcmp order
    std::vector<Attr> attrs;
    // Dataset.
    Type type = Type::U8;
    std::vector<uint64_t> dims;
    bool extendable = false;          // rows kept here and written as 100-row chunks at flush
    std::vector<uint8_t> rows;
    std::vector<uint64_t> chunk_dims; // empty: contiguous
    int gzip = -1;
    uint64_t addr = UNDEF, bytes = 0; // contiguous data
    std::vector<Chunk> chunks;
    // Written by the last flush; a group's B-tree and heap go into its
    // parent's symbol-table entry.  A dataset whose header is written and
    // that has not changed since (every frame, once stored) keeps it.
    uint64_t header = UNDEF, btree = UNDEF, heap = UNDEF;
    bool dirty = true;
    // Extendable datasets: rows stored by the last flush, and how many leading
    // chunks were full then (rows are only appended, so those chunks stay as
    // they are).  Groups: what the last flush wrote them from (member names,
    // member header / B-tree / heap addresses, attributes).
    uint64_t written_rows = UINT64_MAX;
    size_t full_chunks = 0;
    std::string written_as;
};

// A frame for the writer thread: a host row-major copy (host calls), or a
// pinned copy of a device lattice frame already in chunk order (device
// calls, frame_chunks_kernel).
struct FrameJob {
    std::string group, name;          // dataset path
    Type type;
    std::vector<uint64_t> dims;       // [X, Y, Z(, P)]
    std::vector<uint8_t> host;        // host copy (host calls)
    int slot = -1;                    // pinned slot (device calls): the frame in chunk order
};

struct Pinned {
    void *host = nullptr;
    void *dev = nullptr;              // device snapshot of the frame
    size_t bytes = 0;
    bool busy = false;
    cudaEvent_t staged = nullptr;     // snapshot taken (lattice stream)
    cudaEvent_t ready = nullptr;      // host copy done (copy stream)
};

std::string num(uint32_t v, int width)
{
    char b[32];
    snprintf(b, sizeof(b), "%0*u", width, v);
    return b;
}

// The writer's threads run at a lower priority (nice +10) than the thread
// that drives the GPU, so that its wake-ups for the next launch are not
// delayed behind compression.
void lower_priority() { setpriority(PRIO_PROCESS, (id_t)syscall(SYS_gettid), 10); }

// Persistent threads for the chunk work of a frame; the calling thread
// works too.  One parallel loop at a time.
class Pool {
public:
    explicit Pool(unsigned helpers)
    {
        for (unsigned i = 0; i < helpers; i++) th_.emplace_back([this] { loop(); });
    }
    ~Pool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    // Calls fn(i) for i in [0, n) on all threads; returns when every call did.
    void run(size_t n, const std::function<void(size_t)> &fn)
    {
        std::lock_guard<std::mutex> one(run_);
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &fn;
            n_ = n;
            next_ = 0;
            pending_ = th_.size();
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
        fn_ = nullptr;
    }

private:
    void work()
    {
        for (;;) {
            const size_t i = next_++;
            if (i >= n_) break;
            (*fn_)(i);
        }
    }
    void loop()
    {
        lower_priority();
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            lk.unlock();
            work();
            lk.lock();
            if (--pending_ == 0) done_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_, run_;
    std::condition_variable cv_, done_;
    const std::function<void(size_t)> *fn_ = nullptr;
    size_t n_ = 0;
    std::atomic<size_t> next_{0};
    size_t pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

}  // namespace

struct lmb_lmfile {
    int fd = -1;
    std::string path;
    uint64_t eof = SUPERBLOCK;  // relative to the superblock
    Node root;
    // During a flush the metadata is gathered here and written at once.
    bool buffering = false;
    uint64_t pending_at = 0;
    std::vector<uint8_t> pending;
    std::mutex mu;  // tree and file
    int io_error = LMB_OK;
    // Model sizes (loadModel): species for new replicates, the lattice for
    // setDiffusionModelLattice.
    uint32_t number_species = 0;
    uint32_t X = 0, Y = 0, Z = 0, P = 0, bytes_per_particle = 0;
    // Writer thread.
    std::mutex qmu;
    std::condition_variable qcv;
    std::deque<FrameJob> queue;
    int in_flight = 0;
    bool stop = false;
    int error = LMB_OK;
    std::thread writer;
    int device = -1;
    cudaStream_t copy = nullptr;  // device-to-host copies of frames
    Pinned pinned[PINNED_SLOTS];
    uint64_t frames = 0, chunk_bytes = 0;
    std::unique_ptr<Pool> pool;
};

namespace {

// ---- file ------------------------------------------------------------------

bool put(lmb_lmfile *f, uint64_t rel, const void *p, size_t n)
{
    const uint8_t *b = (const uint8_t *)p;
    uint64_t off = USER_BLOCK + rel;
    while (n) {
        const ssize_t w = pwrite(f->fd, b, n, (off_t)off);
        if (w <= 0) {
            f->io_error = LMB_E_IO;
            return false;
        }
        b += w;
        off += (uint64_t)w;
        n -= (size_t)w;
    }
    return true;
}

// Appends at the end of the file; returns the address.
uint64_t append(lmb_lmfile *f, const void *p, size_t n)
{
    const uint64_t a = f->eof;
    if (f->buffering) {
        const uint8_t *b = (const uint8_t *)p;
        f->pending.insert(f->pending.end(), b, b + n);
    } else {
        put(f, a, p, n);
    }
    f->eof += n;
    return a;
}

uint64_t append(lmb_lmfile *f, const Bytes &b) { return append(f, b.v.data(), b.size()); }

// ---- tree ------------------------------------------------------------------

Node *group_at(Node &root, const std::string &path)
{
    Node *n = &root;
    size_t p = 0;
    while (p < path.size()) {
        size_t q = path.find('/', p);
        if (q == std::string::npos) q = path.size();
        const std::string part = path.substr(p, q - p);
        p = q + 1;
        if (part.empty()) continue;
        auto &c = n->children[part];
        if (!c) c.reset(new Node());
        if (!c->group) return nullptr;
        n = c.get();
    }
    return n;
}

// An attribute message must fit a header message's 16-bit size.
bool attr_fits(const Attr &a) { return attribute(a).size() <= 0xFFF8; }

void set_attr(Node &n, Attr a)
{
    for (auto &x : n.attrs)
        if (x.name == a.name) {
            x = std::move(a);
            return;
        }
    n.attrs.push_back(std::move(a));
}

Attr uint_attr(const char *name, uint32_t v)
{
    Attr a{name, Type::U32, 0, {1}, {}};
    for (int i = 0; i < 4; i++) a.data.push_back((uint8_t)(v >> (8 * i)));
    return a;
}

Attr double_attr(const char *name, double v)
{
    Attr a{name, Type::F64, 0, {1}, std::vector<uint8_t>(8)};
    memcpy(a.data.data(), &v, 8);
    return a;
}

Attr string_attr(const std::string &name, const std::string &v)
{
    Attr a{name, Type::STR, (uint32_t)v.size() + 1, {}, {}};
    a.data.assign(v.begin(), v.end());
    a.data.push_back(0);
    return a;
}

// A contiguous dataset whose data is written now (H5LTmake_dataset).
void contiguous(lmb_lmfile *f, Node &g, const std::string &name, Type t, std::vector<uint64_t> dims,
                const void *data)
{
    std::unique_ptr<Node> d(new Node());
    d->group = false;
    d->type = t;
    d->dims = std::move(dims);
    size_t n = type_size(t, 0);
    for (uint64_t x : d->dims) n *= x;
    d->bytes = n;
    d->addr = n ? append(f, data, n) : UNDEF;
    g.children[name] = std::move(d);
}

// An extendable dataset of rows (first dimension unlimited), `rows`-row
// chunks (100 for the reference's own).
Node *extendable_node(Node &g, const std::string &name, Type t, std::vector<uint64_t> dims, uint64_t rows)
{
    auto &c = g.children[name];
    if (!c) {
        c.reset(new Node());
        c->group = false;
        c->type = t;
        c->dims = std::move(dims);
        c->extendable = true;
        c->chunk_dims = c->dims;
        c->chunk_dims[0] = rows;
    }
    return c.get();
}

Node *extendable(Node &g, const std::string &name, Type t, std::vector<uint64_t> dims)
{
    return extendable_node(g, name, t, std::move(dims), ROW_CHUNK);
}

void add_rows(Node &d, const void *p, uint64_t rows)
{
    size_t row = type_size(d.type, 0);
    for (size_t i = 1; i < d.dims.size(); i++) row *= d.dims[i];
    const uint8_t *b = (const uint8_t *)p;
    d.rows.insert(d.rows.end(), b, b + rows * row);
    d.dims[0] += rows;
}

// ---- chunks ----------------------------------------------------------------

// Copies the chunk at `origin` of a row-major array into `dst` (zeroed,
// chunk-shaped).  Trailing dimensions that the chunk spans whole are merged
// with the one before them, so each copied run is as long as both layouts
// allow (a lattice frame's z column with all its slots, for instance).
void gather_chunk(const uint8_t *src, const std::vector<uint64_t> &dims0, const std::vector<uint64_t> &cd0,
                  const std::vector<uint64_t> &origin0, size_t esize, uint8_t *dst)
{
    std::vector<uint64_t> dims = dims0, cd = cd0, origin = origin0;
    while (dims.size() > 1 && cd.back() == dims.back() && origin.back() == 0) {
        const uint64_t n = dims.back();
        dims.pop_back();
        cd.pop_back();
        origin.pop_back();
        dims.back() *= n;
        cd.back() *= n;
        origin.back() *= n;
    }
    const size_t r = dims.size();
    std::vector<uint64_t> ss(r), ds(r), ext(r), idx(r, 0);
    ss[r - 1] = ds[r - 1] = 1;
    for (int i = (int)r - 2; i >= 0; i--) {
        ss[i] = ss[i + 1] * dims[i + 1];
        ds[i] = ds[i + 1] * cd[i + 1];
    }
    for (size_t i = 0; i < r; i++) ext[i] = std::min(cd[i], dims[i] - origin[i]);
    const size_t run = ext[r - 1] * esize;
    for (;;) {
        uint64_t so = 0, doff = 0;
        for (size_t i = 0; i < r; i++) {
            so += (origin[i] + idx[i]) * ss[i];
            doff += idx[i] * ds[i];
        }
        memcpy(dst + doff * esize, src + so * esize, run);
        int i = (int)r - 2;
        while (i >= 0) {
            if (++idx[i] < ext[i]) break;
            idx[i] = 0;
            i--;
        }
        if (i < 0) break;
    }
}

// Splits a row-major array into chunks (in lexicographic chunk order, the
// order the chunk B-tree keeps), gzipped when level >= 0, on `threads`
// threads.  Returns false when zlib fails.
using Gather = std::function<void(const std::vector<uint64_t> &origin, uint8_t *dst)>;

// zlib's compress2 with a stream kept per thread: deflateInit's defaults
// (zlib format, 32 KB window, memory level 8, default strategy) give the
// same bytes, without allocating and clearing the stream for every chunk.
struct Deflater {
    z_stream s{};
    int level = -1;
    ~Deflater()
    {
        if (level >= 0) deflateEnd(&s);
    }
    std::vector<uint8_t> scratch;  // deflateBound-sized, reused: only the result is copied out
    bool run(const uint8_t *in, size_t n, int lvl, std::vector<uint8_t> &out)
    {
        if (level != lvl) {
            if (level >= 0) deflateEnd(&s);
            s = z_stream{};
            level = -1;
            if (deflateInit(&s, lvl) != Z_OK) return false;
            level = lvl;
        } else if (deflateReset(&s) != Z_OK) {
            return false;
        }
        const size_t bound = deflateBound(&s, n);
        if (scratch.size() < bound) scratch.resize(bound);
        s.next_in = const_cast<Bytef *>(in);
        s.avail_in = (uInt)n;
        s.next_out = scratch.data();
        s.avail_out = (uInt)bound;
        if (deflate(&s, Z_FINISH) != Z_STREAM_END) return false;
        out.assign(scratch.data(), scratch.data() + (bound - s.avail_out));
        return true;
    }
};

// `direct`, when given, holds the chunks already in chunk order, each
// contiguous: they are compressed where they lie.
bool make_chunks(const Gather &gather, const std::vector<uint64_t> &dims, const std::vector<uint64_t> &cd,
                 size_t esize, int level, Pool &pool, std::vector<std::vector<uint8_t>> &out,
                 std::vector<std::vector<uint64_t>> &origins, const uint8_t *direct = nullptr)
{
    const size_t r = dims.size();
    std::vector<uint64_t> grid(r);
    size_t nch = 1, celems = 1;
    for (size_t i = 0; i < r; i++) {
        if (dims[i] == 0 || cd[i] == 0 || cd[i] > dims[i]) return false;
        grid[i] = (dims[i] + cd[i] - 1) / cd[i];
        nch *= grid[i];
        celems *= cd[i];
    }
    out.assign(nch, {});
    origins.assign(nch, std::vector<uint64_t>(r));
    for (size_t c = 0; c < nch; c++) {
        size_t rem = c;
        for (int i = (int)r - 1; i >= 0; i--) {
            origins[c][i] = (rem % grid[i]) * cd[i];
            rem /= grid[i];
        }
    }
    const size_t cbytes = celems * esize;
    std::atomic<bool> ok{true};
    pool.run(nch, [&](size_t c) {
        thread_local std::vector<uint8_t> raw;
        const uint8_t *in = direct ? direct + c * cbytes : nullptr;
        if (!in) {
            raw.assign(cbytes, 0);
            gather(origins[c], raw.data());
            in = raw.data();
        }
        if (level < 0) {
            out[c].assign(in, in + cbytes);
            return;
        }
        thread_local Deflater z;
        if (!z.run(in, cbytes, level, out[c])) ok = false;
    });
    return ok;
}

// A chunked dataset from a row-major array (writeParticleLattice_U8LE and
// friends): chunks are compressed outside the file lock, then appended.
int chunked_dataset(lmb_lmfile *f, const std::string &group, const std::string &name, Type t,
                    const std::vector<uint64_t> &dims, const std::vector<uint64_t> &cd, int level,
                    const Gather &gather, const uint8_t *direct = nullptr)
{
    std::vector<std::vector<uint8_t>> out;
    std::vector<std::vector<uint64_t>> origins;
    if (!make_chunks(gather, dims, cd, type_size(t, 0), level, *f->pool, out, origins, direct)) return LMB_E_IO;
    std::lock_guard<std::mutex> lk(f->mu);
    std::unique_ptr<Node> d(new Node());
    d->group = false;
    d->type = t;
    d->dims = dims;
    d->chunk_dims = cd;
    d->gzip = level;
    // The chunks back to back, in one write.
    std::vector<uint8_t> all;
    for (auto &o : out) all.insert(all.end(), o.begin(), o.end());
    const uint64_t base = append(f, all.data(), all.size());
    uint64_t total = 0;
    for (size_t c = 0; c < out.size(); c++) {
        d->chunks.push_back({origins[c], base + total, (uint32_t)out[c].size()});
        total += out[c].size();
    }
    Node *g = group_at(f->root, group);
    if (!g) return LMB_E_STATE;
    g->children[name] = std::move(d);
    f->chunk_bytes += total;
    return f->io_error;
}

int chunked_dataset(lmb_lmfile *f, const std::string &group, const std::string &name, Type t,
                    const std::vector<uint64_t> &dims, const std::vector<uint64_t> &cd, int level,
                    const uint8_t *row_major)
{
    const size_t esize = type_size(t, 0);
    return chunked_dataset(f, group, name, t, dims, cd, level,
                           [&](const std::vector<uint64_t> &o, uint8_t *dst) {
                               gather_chunk(row_major, dims, cd, o, esize, dst);
                           });
}

// A device lattice frame written straight into chunk order: chunk c =
// (cx * gy + cy) * gz + cz of cx x cy x cz sites (x slowest), each chunk
// [xx][yy][zz][p] contiguous (the layout its HDF5 chunk stores), so that the
// host only compresses.  One thread per native word (ByteLattice: 4 slots,
// IntLattice: 1 slot) or per site type; consecutive threads read
// consecutive sites of one word plane.  Positions of edge chunks beyond the
// lattice are left as they are (zeroed before the launch).
struct ChunkShape {
    uint32_t X, Y, Z, P, cx, cy, cz, gy, gz;
};

__global__ void frame_chunks_kernel(const uint32_t *__restrict__ native, const uint8_t *__restrict__ sites,
                                    uint8_t *__restrict__ out, ChunkShape k, uint32_t words, uint32_t bps)
{
    const uint64_t N = (uint64_t)k.X * k.Y * k.Z;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * (sites ? 1 : words)) return;
    const uint64_t i = t % N, w = t / N;
    const uint32_t x = (uint32_t)(i % k.X), y = (uint32_t)((i / k.X) % k.Y), z = (uint32_t)(i / ((uint64_t)k.X * k.Y));
    const uint32_t bx = x / k.cx, by = y / k.cy, bz = z / k.cz;
    const uint64_t c = ((uint64_t)bx * k.gy + by) * k.gz + bz;
    const uint64_t e = ((uint64_t)(x - bx * k.cx) * k.cy + (y - by * k.cy)) * k.cz + (z - bz * k.cz);
    const uint64_t cell = (uint64_t)k.cx * k.cy * k.cz;
    if (sites) {
        out[c * cell + e] = sites[i];
    } else {
        const uint64_t cb = cell * k.P * bps;  // chunk bytes
        const uint64_t off = c * cb + (bps == 1 ? e * k.P + 4 * w : (e * k.P + w) * 4);
        *(uint32_t *)(out + off) = native[w * N + i];
    }
}

// ---- metadata --------------------------------------------------------------

struct Item {
    uint64_t addr;
    Bytes lo, hi;  // encoded keys bounding the child
};

// Version-1 B-tree over `items` (in key order), built bottom-up with full
// nodes; returns the root's address.  Every node is allocated at the size
// libhdf5 reads (2K children, 2K + 1 keys).
uint64_t btree(lmb_lmfile *f, int type, std::vector<Item> items, size_t key_size, uint32_t K,
               const Bytes &empty_key)
{
    const size_t fan = 2 * K;
    const size_t node = 24 + (2 * K + 1) * key_size + 2 * K * 8;
    if (items.empty()) {
        Bytes b;
        b.raw("TREE", 4);
        b.u8(type);
        b.u8(0);
        b.u16(0);
        b.u64(UNDEF);
        b.u64(UNDEF);
        b.raw(empty_key);
        b.zeros(node - b.size());
        return append(f, b);
    }
    for (int level = 0;; level++) {
        const size_t nn = (items.size() + fan - 1) / fan;
        const uint64_t base = f->eof;
        Bytes all;
        std::vector<Item> up;
        for (size_t j = 0; j < nn; j++) {
            const size_t a = j * fan, e = std::min(a + fan, items.size());
            Bytes b;
            b.raw("TREE", 4);
            b.u8(type);
            b.u8(level);
            b.u16(e - a);
            b.u64(j ? base + (j - 1) * node : UNDEF);
            b.u64(j + 1 < nn ? base + (j + 1) * node : UNDEF);
            for (size_t i = a; i < e; i++) {
                b.raw(items[i].lo);
                b.u64(items[i].addr);
            }
            b.raw(items[e - 1].hi);
            b.zeros(node - b.size());
            all.raw(b);
            up.push_back({base + j * node, items[a].lo, items[e - 1].hi});
        }
        append(f, all);
        if (nn == 1) return base;
        items = std::move(up);
    }
}

Bytes chunk_key(uint32_t nbytes, const std::vector<uint64_t> &off, uint64_t last)
{
    Bytes k;
    k.u32(nbytes);
    k.u32(0);  // filter mask: every filter applied
    for (uint64_t o : off) k.u64(o);
    k.u64(last);
    return k;
}

uint64_t header(lmb_lmfile *f, const std::vector<std::pair<uint16_t, Bytes>> &msgs)
{
    Bytes body;
    for (auto &m : msgs) {
        Bytes d = m.second;
        d.pad8();
        if (d.size() > 0xFFFF) f->io_error = LMB_E_ARG;
        body.u16(m.first);
        body.u16(d.size());
        body.u8(m.first == 0x0003 || m.first == 0x0005 ? 1 : 0);  // constant: datatype, fill value
        body.zeros(3);
        body.raw(d);
    }
    Bytes h;
    h.u8(1);
    h.u8(0);
    h.u16(msgs.size());
    h.u32(1);
    h.u32(body.size());
    h.u32(0);
    h.raw(body);
    return append(f, h);
}

void write_node(lmb_lmfile *f, Node &n);

// A group is written again only when a member was added or rewritten (its
// header, B-tree or heap moved) or an attribute changed; otherwise its header,
// heap and B-tree stay where the last flush put them.
void write_group(lmb_lmfile *f, Node &g)
{
    for (auto &c : g.children) write_node(f, *c.second);
    std::string as;
    for (auto &c : g.children) {
        as += c.first;
        as.push_back('\0');
        const uint64_t a[3] = {c.second->header, c.second->btree, c.second->heap};
        as.append((const char *)a, sizeof a);
    }
    for (auto &a : g.attrs) {
        const Bytes b = attribute(a);
        as.append((const char *)b.v.data(), b.size());
    }
    if (g.header != UNDEF && as == g.written_as) return;
    g.written_as = std::move(as);
    // Local heap: "" at offset 0, then each name, 8-byte aligned.
    Bytes data;
    data.zeros(8);
    std::vector<uint64_t> offs;
    for (auto &c : g.children) {
        offs.push_back(data.size());
        data.raw(c.first.c_str(), c.first.size() + 1);
        data.pad8();
    }
    Bytes heap;
    heap.raw("HEAP", 4);
    heap.zeros(4);
    heap.u64(data.size());
    heap.u64(1);  // no free block
    heap.u64(f->eof + 32);
    heap.raw(data);
    g.heap = append(f, heap);
    // Symbol-table nodes of up to 2 * SYM_LEAF_K entries, in name order.
    std::vector<Item> items;
    const size_t per = 2 * SYM_LEAF_K, snod = 8 + per * 40;
    size_t i = 0;
    uint64_t prev_hi = 0;
    std::vector<Node *> kids;
    for (auto &c : g.children) kids.push_back(c.second.get());
    while (i < kids.size()) {
        const size_t e = std::min(i + per, kids.size());
        Bytes b;
        b.raw("SNOD", 4);
        b.u8(1);
        b.u8(0);
        b.u16(e - i);
        for (size_t k = i; k < e; k++) {
            Node *c = kids[k];
            b.u64(offs[k]);
            b.u64(c->header);
            b.u32(c->group ? 1 : 0);
            b.u32(0);
            b.u64(c->group ? c->btree : 0);
            b.u64(c->group ? c->heap : 0);
        }
        b.zeros(snod - b.size());
        Item it;
        it.addr = append(f, b);
        it.lo.u64(prev_hi);
        it.hi.u64(offs[e - 1]);
        prev_hi = offs[e - 1];
        items.push_back(std::move(it));
        i = e;
    }
    Bytes zero;
    zero.u64(0);
    g.btree = btree(f, 0, std::move(items), 8, BTREE_K, zero);
    std::vector<std::pair<uint16_t, Bytes>> msgs;
    Bytes stab;
    stab.u64(g.btree);
    stab.u64(g.heap);
    msgs.push_back({0x0011, stab});
    for (auto &a : g.attrs) msgs.push_back({0x000C, attribute(a)});
    g.header = header(f, msgs);
}

void write_dataset(lmb_lmfile *f, Node &d)
{
    if (!d.dirty && d.header != UNDEF && (!d.extendable || d.written_rows == d.dims[0])) return;
    d.dirty = false;
    const size_t esize = type_size(d.type, 0);
    if (d.extendable) {
        // The rows, in 100-row chunks (the last one zero-filled), uncompressed.
        size_t row = esize;
        for (size_t i = 1; i < d.dims.size(); i++) row *= d.dims[i];
        // (Chunks span whole rows: a copied dataset chunked across its
        // other dimensions is stored with full-width chunks.)
        for (size_t i = 1; i < d.dims.size(); i++) d.chunk_dims[i] = std::max<uint64_t>(1, d.dims[i]);
        const uint64_t per = d.chunk_dims[0];
        // Chunks that were full at an earlier flush are kept; the partial
        // last one and any new ones are appended.
        if (d.full_chunks > d.chunks.size()) d.full_chunks = d.chunks.size();
        d.chunks.resize(d.full_chunks);
        std::vector<uint8_t> buf(per * row);
        for (uint64_t r0 = d.full_chunks * per; r0 < d.dims[0]; r0 += per) {
            std::fill(buf.begin(), buf.end(), 0);
            const uint64_t n = std::min<uint64_t>(per, d.dims[0] - r0);
            memcpy(buf.data(), d.rows.data() + r0 * row, n * row);
            std::vector<uint64_t> off(d.dims.size(), 0);
            off[0] = r0;
            d.chunks.push_back({off, append(f, buf.data(), buf.size()), (uint32_t)buf.size()});
        }
        d.full_chunks = (size_t)(d.dims[0] / per);
        d.written_rows = d.dims[0];
    }
    std::vector<std::pair<uint16_t, Bytes>> msgs;
    msgs.push_back({0x0001, dataspace(d.dims, d.extendable)});
    msgs.push_back({0x0003, datatype(d.type)});
    Bytes fill;
    fill.u8(2);
    fill.u8(d.chunk_dims.empty() ? 2 : 3);  // allocation: late (contiguous), incremental (chunked)
    fill.u8(2);                             // fill written if set
    fill.u8(1);                             // defined, of size 0: the default (zeros)
    fill.u32(0);
    msgs.push_back({0x0005, fill});
    Bytes lay;
    lay.u8(3);
    if (d.chunk_dims.empty()) {
        lay.u8(1);
        lay.u64(d.addr);
        lay.u64(d.bytes);
    } else {
        const size_t rank = d.dims.size();
        uint64_t root = UNDEF;
        if (!d.chunks.empty()) {
            std::vector<Item> items;
            for (size_t c = 0; c < d.chunks.size(); c++) {
                Item it;
                it.addr = d.chunks[c].addr;
                it.lo = chunk_key(d.chunks[c].nbytes, d.chunks[c].offset, 0);
                if (c + 1 < d.chunks.size()) {
                    it.hi = chunk_key(d.chunks[c + 1].nbytes, d.chunks[c + 1].offset, 0);
                } else {
                    std::vector<uint64_t> end(rank);
                    for (size_t k = 0; k < rank; k++) end[k] = d.chunks[c].offset[k] + d.chunk_dims[k];
                    it.hi = chunk_key(0, end, esize);
                }
                items.push_back(std::move(it));
            }
            root = btree(f, 1, std::move(items), 8 + 8 * (rank + 1), ISTORE_K, Bytes());
        }
        lay.u8(2);
        lay.u8(rank + 1);
        lay.u64(root);
        for (uint64_t c : d.chunk_dims) lay.u32(c);
        lay.u32(esize);
    }
    msgs.push_back({0x0008, lay});
    if (d.gzip >= 0) {
        Bytes fp;
        fp.u8(1);
        fp.u8(1);
        fp.zeros(6);
        fp.u16(1);  // deflate
        fp.u16(8);
        fp.u16(1);  // optional, as H5Pset_deflate adds it
        fp.u16(1);
        fp.raw("deflate\0", 8);
        fp.u32(d.gzip);
        fp.u32(0);
        msgs.push_back({0x000B, fp});
    }
    for (auto &a : d.attrs) msgs.push_back({0x000C, attribute(a)});
    d.header = header(f, msgs);
}

void write_node(lmb_lmfile *f, Node &n)
{
    if (n.group) write_group(f, n);
    else write_dataset(f, n);
}

// Writes the metadata and points the superblock at it (caller holds mu).
int commit(lmb_lmfile *f)
{
    f->buffering = true;
    f->pending.clear();
    f->pending_at = f->eof;
    write_node(f, f->root);
    f->buffering = false;
    if (!f->pending.empty()) put(f, f->pending_at, f->pending.data(), f->pending.size());
    f->pending.clear();
    f->pending.shrink_to_fit();
    Bytes sb;
    sb.raw("\x89HDF\r\n\x1a\n", 8);
    sb.u8(0);  // superblock version
    sb.u8(0);  // free-space version
    sb.u8(0);  // root group symbol-table entry version
    sb.u8(0);
    sb.u8(0);  // shared header message format version
    sb.u8(8);  // size of offsets
    sb.u8(8);  // size of lengths
    sb.u8(0);
    sb.u16(SYM_LEAF_K);
    sb.u16(BTREE_K);
    sb.u32(0);
    sb.u64(USER_BLOCK);            // base address: the superblock's own
    sb.u64(UNDEF);                 // free-space info
    sb.u64(USER_BLOCK + f->eof);   // end of file (absolute)
    sb.u64(UNDEF);                 // driver info
    sb.u64(0);                     // root entry: link name offset
    sb.u64(f->root.header);
    sb.u32(1);
    sb.u32(0);
    sb.u64(f->root.btree);
    sb.u64(f->root.heap);
    put(f, 0, sb.v.data(), sb.size());
    if (ftruncate(f->fd, (off_t)(USER_BLOCK + f->eof)) != 0) f->io_error = LMB_E_IO;
    return f->io_error;
}

// ---- replicates ------------------------------------------------------------

// SimulationFile::createReplicateHandles (SimulationFile.cpp:2187-2226).
Node *replicate(lmb_lmfile *f, uint32_t rep)
{
    Node *g = group_at(f->root, "Simulations/" + num(rep, 7));
    if (g && !g->children.count("SpeciesCounts")) {
        extendable(*g, "SpeciesCounts", Type::I32, {0, f->number_species});
        extendable(*g, "SpeciesCountTimes", Type::F64, {0});
    }
    return g;
}

// Appends a time to Lattice/LatticeTimes or Sites/SiteTimes; returns the
// frame index (SimulationFile.cpp:1198-1230).
uint32_t next_frame(lmb_lmfile *f, uint32_t rep, const char *group, const char *times, double t)
{
    Node *g = replicate(f, rep);
    group_at(*g, group);
    Node *d = extendable(*g, times, Type::F64, {0});
    const uint32_t index = (uint32_t)d->dims[0];
    add_rows(*d, &t, 1);
    return index;
}

void writer_main(lmb_lmfile *f)
{
    lower_priority();
    for (;;) {
        FrameJob j;
        {
            std::unique_lock<std::mutex> lk(f->qmu);
            f->qcv.wait(lk, [&] { return f->stop || !f->queue.empty(); });
            if (f->queue.empty()) return;
            j = std::move(f->queue.front());
            f->queue.pop_front();
        }
        int rc = LMB_OK;
        const uint8_t *data = j.host.data();
        if (j.slot >= 0) {
            cudaSetDevice(f->device);
            if (cudaEventSynchronize(f->pinned[j.slot].ready) != cudaSuccess) rc = LMB_E_CUDA;
            data = (const uint8_t *)f->pinned[j.slot].host;
        }
        if (rc == LMB_OK) {
            std::vector<uint64_t> cd(j.dims.size());
            for (size_t i = 0; i < cd.size(); i++) cd[i] = i < 3 ? std::min(FRAME_CHUNK, j.dims[i]) : j.dims[i];
            if (j.slot >= 0) {
                // Already in chunk order (frame_chunks_kernel): compressed in place.
                rc = chunked_dataset(f, j.group, j.name, j.type, j.dims, cd, FRAME_GZIP,
                                     [](const std::vector<uint64_t> &, uint8_t *) {}, data);
            } else {
                rc = chunked_dataset(f, j.group, j.name, j.type, j.dims, cd, FRAME_GZIP, data);
            }
        }
        if (rc == LMB_OK) {
            std::lock_guard<std::mutex> lk(f->mu);
            f->frames++;
        }
        {
            std::lock_guard<std::mutex> lk(f->qmu);
            if (j.slot >= 0) f->pinned[j.slot].busy = false;
            f->in_flight--;
            if (rc != LMB_OK && f->error == LMB_OK) f->error = rc;
        }
        f->qcv.notify_all();
    }
}

void push(lmb_lmfile *f, FrameJob &&j)
{
    {
        std::lock_guard<std::mutex> lk(f->qmu);
        f->queue.push_back(std::move(j));
        f->in_flight++;
    }
    f->qcv.notify_all();
}

int status(lmb_lmfile *f)
{
    std::lock_guard<std::mutex> lk(f->qmu);
    return f->error;
}

int drain(lmb_lmfile *f)
{
    std::unique_lock<std::mutex> lk(f->qmu);
    f->qcv.wait(lk, [&] { return f->in_flight == 0; });
    return f->error;
}

// A free pinned slot with room for `bytes` on the file's device (waits for
// the writer thread to release one).
int take_slot(lmb_lmfile *f, size_t bytes, int *slot)
{
    std::unique_lock<std::mutex> lk(f->qmu);
    f->qcv.wait(lk, [&] {
        if (f->error != LMB_OK) return true;
        for (auto &p : f->pinned)
            if (!p.busy) return true;
        return false;
    });
    if (f->error != LMB_OK) return f->error;
    for (int s = 0; s < PINNED_SLOTS; s++) {
        Pinned &p = f->pinned[s];
        if (p.busy) continue;
        if (p.bytes < bytes) {
            if (p.host) cudaFreeHost(p.host);
            if (p.dev) cudaFree(p.dev);
            p.host = p.dev = nullptr;
            p.bytes = 0;
            if (cudaMallocHost(&p.host, bytes) != cudaSuccess) return LMB_E_NOMEM;
            if (cudaMalloc(&p.dev, bytes) != cudaSuccess) return LMB_E_NOMEM;
            p.bytes = bytes;
        }
        if (!p.ready && cudaEventCreateWithFlags(&p.ready, cudaEventDisableTiming) != cudaSuccess)
            return LMB_E_CUDA;
        if (!p.staged && cudaEventCreateWithFlags(&p.staged, cudaEventDisableTiming) != cudaSuccess)
            return LMB_E_CUDA;
        p.busy = true;
        *slot = s;
        return LMB_OK;
    }
    return LMB_E_STATE;
}

int append_device(lmb_lmfile *f, uint32_t rep, double time, lmb_lattice *lat, bool sites)
{
    lmb::LatticeView v;
    if (!f || lmb::lattice_view(lat, &v) != LMB_OK) return LMB_E_ARG;
    if (v.pending) return LMB_E_STATE;
    int rc = status(f);
    if (rc != LMB_OK) return rc;
    if (f->device < 0) f->device = v.ctx->device;
    if (f->device != v.ctx->device) return LMB_E_ARG;
    if (cudaSetDevice(f->device) != cudaSuccess) return LMB_E_CUDA;
    const size_t N = v.g.N, esize = v.bytes_per_slot;
    ChunkShape k;
    k.X = v.g.X;
    k.Y = v.g.Y;
    k.Z = v.g.Z;
    k.P = sites ? 1 : v.slots;
    k.cx = (uint32_t)std::min<uint64_t>(FRAME_CHUNK, k.X);
    k.cy = (uint32_t)std::min<uint64_t>(FRAME_CHUNK, k.Y);
    k.cz = (uint32_t)std::min<uint64_t>(FRAME_CHUNK, k.Z);
    const uint32_t gx = (k.X + k.cx - 1) / k.cx;
    k.gy = (k.Y + k.cy - 1) / k.cy;
    k.gz = (k.Z + k.cz - 1) / k.cz;
    const bool ragged = k.X % k.cx || k.Y % k.cy || k.Z % k.cz;
    const size_t bytes = (size_t)gx * k.gy * k.gz * k.cx * k.cy * k.cz * k.P * (sites ? 1 : esize);
    const uint32_t words = esize == 1 ? v.slots / 4 : v.slots;
    if (!f->copy && cudaStreamCreateWithFlags(&f->copy, cudaStreamNonBlocking) != cudaSuccess) return LMB_E_CUDA;
    int s = -1;
    rc = take_slot(f, bytes, &s);
    if (rc != LMB_OK) return rc;
    Pinned &p = f->pinned[s];
    // The frame in chunk order, in the lattice's stream order (the lattice
    // may be advanced right after), then the copy to pinned memory on the
    // file's own stream, overlapping the next timesteps.
    cudaStream_t st = v.ctx->stream;
    cudaError_t e = ragged ? cudaMemsetAsync(p.dev, 0, bytes, st) : cudaSuccess;
    if (e == cudaSuccess) {
        const uint64_t threads = (uint64_t)N * (sites ? 1 : words);
        frame_chunks_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
            v.particles, sites ? v.sites : nullptr, (uint8_t *)p.dev, k, words, (uint32_t)esize);
        lmb::count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(p.staged, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(f->copy, p.staged, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p.host, p.dev, bytes, cudaMemcpyDeviceToHost, f->copy);
    if (e == cudaSuccess) e = cudaEventRecord(p.ready, f->copy);
    if (e != cudaSuccess) {
        // Work already queued on either stream may still write the slot's
        // buffers: wait for both streams before the slot is handed out again,
        // and wake a thread waiting for a free slot.
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(f->copy);
        {
            std::lock_guard<std::mutex> lk(f->qmu);
            p.busy = false;
        }
        f->qcv.notify_all();
        return LMB_E_CUDA;
    }
    FrameJob j;
    j.slot = s;
    {
        std::lock_guard<std::mutex> lk(f->mu);
        const char *grp = sites ? "Sites" : "Lattice";
        const uint32_t index = next_frame(f, rep, grp, sites ? "SiteTimes" : "LatticeTimes", time);
        j.group = "Simulations/" + num(rep, 7) + "/" + grp;
        j.name = num(index, 10);
    }
    if (sites) {
        j.type = Type::U8;
        j.dims = {v.g.X, v.g.Y, v.g.Z};
    } else {
        j.type = esize == 1 ? Type::U8 : Type::U32;
        j.dims = {v.g.X, v.g.Y, v.g.Z, v.slots};
    }
    push(f, std::move(j));
    return LMB_OK;
}

}  // namespace

// ---- C ABI -------------------------------------------------------------------

extern "C" int lmb_lmfile_create(const char *path, lmb_lmfile **out)
{
    if (!path || !out) return LMB_E_ARG;
    *out = nullptr;
    const int fd = open(path, O_RDWR | O_CREAT | O_EXCL, 0644);
    if (fd < 0) return LMB_E_IO;
    lmb_lmfile *f = new lmb_lmfile();
    f->fd = fd;
    f->path = path;
    // Chunk compression threads: up to 16, leaving two host cores to the
    // thread that drives the GPU; LMB_LMFILE_THREADS sets the number.
    const unsigned hw = std::thread::hardware_concurrency();
    unsigned nt = std::max(1u, std::min(16u, hw > 2 ? hw - 2 : 1u));
    if (const char *e = getenv("LMB_LMFILE_THREADS")) {
        const int v = atoi(e);
        if (v >= 1 && v <= 256) nt = (unsigned)v;
    }
    f->pool.reset(new Pool(nt - 1));
    // The user block: "LMH5" and zeros (SimulationFile_create.cpp:119-128).
    const uint8_t ub[USER_BLOCK] = {'L', 'M', 'H', '5'};
    if (pwrite(fd, ub, sizeof(ub), 0) != (ssize_t)sizeof(ub)) f->io_error = LMB_E_IO;
    set_attr(f->root, uint_attr("formatVersion", FORMAT_VERSION));
    group_at(f->root, "Parameters");
    group_at(f->root, "Model");
    group_at(f->root, "Simulations");
    int rc;
    {
        std::lock_guard<std::mutex> lk(f->mu);
        rc = commit(f);
    }
    if (rc != LMB_OK) {
        close(fd);
        delete f;
        return rc;
    }
    f->writer = std::thread(writer_main, f);
    *out = f;
    return LMB_OK;
}

extern "C" int lmb_lmfile_set_parameter(lmb_lmfile *f, const char *key, const char *value)
{
    if (!f || !key || !value || !*key) return LMB_E_ARG;
    Attr a = string_attr(key, value);
    if (!attr_fits(a)) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    set_attr(*group_at(f->root, "Parameters"), std::move(a));
    return f->io_error;
}

extern "C" int lmb_lmfile_set_reaction_model(lmb_lmfile *f, uint32_t ns, uint32_t nr, const uint32_t *init,
                                             const uint32_t *types, const double *k, const double *noise,
                                             const int32_t *S, const uint32_t *D)
{
    if (!f || !init || (nr && (!types || !k || !S || !D))) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    Node *model = group_at(f->root, "Model");
    model->children.erase("Reaction");
    Node *g = group_at(*model, "Reaction");
    f->number_species = ns;
    set_attr(*g, uint_attr("numberSpecies", ns));
    set_attr(*g, uint_attr("numberReactions", nr));
    contiguous(f, *g, "InitialSpeciesCounts", Type::U32, {ns}, init);
    if (nr) {
        contiguous(f, *g, "ReactionTypes", Type::U32, {nr}, types);
        contiguous(f, *g, "ReactionRateConstants", Type::F64, {nr, 10}, k);
        if (noise) contiguous(f, *g, "ReactionRateNoise", Type::F64, {nr, 2}, noise);
        contiguous(f, *g, "StoichiometricMatrix", Type::I32, {ns, nr}, S);
        contiguous(f, *g, "DependencyMatrix", Type::U32, {ns, nr}, D);
    }
    return f->io_error;
}

extern "C" int lmb_lmfile_set_diffusion_model(lmb_lmfile *f, uint32_t ns, uint32_t nr, uint32_t nst,
                                              double spacing, uint32_t X, uint32_t Y, uint32_t Z, uint32_t P,
                                              uint32_t bpp, const double *DF, const uint32_t *RL)
{
    if (!f || !DF || (nr && !RL) || !ns || !nst || !(spacing > 0.0) || !X || !Y || !Z || !P ||
        (bpp != 1 && bpp != 4))
        return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    Node *model = group_at(f->root, "Model");
    model->children.erase("Diffusion");
    Node *g = group_at(*model, "Diffusion");
    f->number_species = ns;
    f->X = X;
    f->Y = Y;
    f->Z = Z;
    f->P = P;
    f->bytes_per_particle = bpp;
    set_attr(*g, uint_attr("numberSpecies", ns));
    set_attr(*g, uint_attr("numberReactions", nr));
    set_attr(*g, uint_attr("numberSiteTypes", nst));
    set_attr(*g, double_attr("latticeSpacing", spacing));
    set_attr(*g, uint_attr("latticeXSize", X));
    set_attr(*g, uint_attr("latticeYSize", Y));
    set_attr(*g, uint_attr("latticeZSize", Z));
    set_attr(*g, uint_attr("particlesPerSite", P));
    set_attr(*g, uint_attr("bytes_per_particle", bpp));
    contiguous(f, *g, "DiffusionMatrix", Type::F64, {nst, nst, ns}, DF);
    if (nr) contiguous(f, *g, "ReactionLocationMatrix", Type::U32, {nr, nst}, RL);
    return f->io_error;
}

extern "C" int lmb_lmfile_set_diffusion_model_lattice(lmb_lmfile *f, const void *particles, const uint8_t *sites)
{
    if (!f || !particles || !sites) return LMB_E_ARG;
    if (!f->X) return LMB_E_STATE;
    const std::vector<uint64_t> dims = {f->X, f->Y, f->Z, f->P};
    const std::vector<uint64_t> cd = {std::min<uint64_t>(FRAME_CHUNK, f->X), std::min<uint64_t>(FRAME_CHUNK, f->Y),
                                      std::min<uint64_t>(FRAME_CHUNK, f->Z), f->P};
    int rc = chunked_dataset(f, "Model/Diffusion", "Lattice", f->bytes_per_particle == 1 ? Type::U8 : Type::U32,
                             dims, cd, FRAME_GZIP, (const uint8_t *)particles);
    if (rc != LMB_OK) return rc;
    return chunked_dataset(f, "Model/Diffusion", "LatticeSites", Type::U8, {f->X, f->Y, f->Z}, {cd[0], cd[1], cd[2]},
                           FRAME_GZIP, sites);
}

extern "C" int lmb_lmfile_append_species_counts(lmb_lmfile *f, uint32_t rep, uint32_t rows, uint32_t ns,
                                                const double *times, const int32_t *counts)
{
    if (!f || (rows && (!times || !counts))) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    Node *g = replicate(f, rep);
    Node *c = g->children["SpeciesCounts"].get();
    Node *t = g->children["SpeciesCountTimes"].get();
    if (c->dims[0] == 0) c->dims[1] = ns;
    if (c->dims[1] != ns) return LMB_E_ARG;
    add_rows(*c, counts, rows);
    add_rows(*t, times, rows);
    c->chunk_dims[1] = ns;
    return f->io_error;
}

extern "C" int lmb_lmfile_append_lattice(lmb_lmfile *f, uint32_t rep, double time, uint32_t X, uint32_t Y,
                                         uint32_t Z, uint32_t P, uint32_t bpp, const void *particles)
{
    if (!f || !particles || !X || !Y || !Z || !P || (bpp != 1 && bpp != 4)) return LMB_E_ARG;
    int rc = status(f);
    if (rc != LMB_OK) return rc;
    FrameJob j;
    j.type = bpp == 1 ? Type::U8 : Type::U32;
    j.dims = {X, Y, Z, P};
    const uint8_t *b = (const uint8_t *)particles;
    j.host.assign(b, b + (size_t)X * Y * Z * P * bpp);
    {
        std::lock_guard<std::mutex> lk(f->mu);
        const uint32_t index = next_frame(f, rep, "Lattice", "LatticeTimes", time);
        j.group = "Simulations/" + num(rep, 7) + "/Lattice";
        j.name = num(index, 10);
    }
    push(f, std::move(j));
    return LMB_OK;
}

extern "C" int lmb_lmfile_append_lattice_device(lmb_lmfile *f, uint32_t rep, double time, lmb_lattice *lattice)
{
    return append_device(f, rep, time, lattice, false);
}

extern "C" int lmb_lmfile_append_sites(lmb_lmfile *f, uint32_t rep, double time, uint32_t X, uint32_t Y,
                                       uint32_t Z, const uint8_t *sites)
{
    if (!f || !sites || !X || !Y || !Z) return LMB_E_ARG;
    int rc = status(f);
    if (rc != LMB_OK) return rc;
    FrameJob j;
    j.type = Type::U8;
    j.dims = {X, Y, Z};
    j.host.assign(sites, sites + (size_t)X * Y * Z);
    {
        std::lock_guard<std::mutex> lk(f->mu);
        const uint32_t index = next_frame(f, rep, "Sites", "SiteTimes", time);
        j.group = "Simulations/" + num(rep, 7) + "/Sites";
        j.name = num(index, 10);
    }
    push(f, std::move(j));
    return LMB_OK;
}

extern "C" int lmb_lmfile_append_sites_device(lmb_lmfile *f, uint32_t rep, double time, lmb_lattice *lattice)
{
    return append_device(f, rep, time, lattice, true);
}

extern "C" int lmb_lmfile_write_max_counts(lmb_lmfile *f, uint32_t rep, const uint32_t *mp, uint32_t np,
                                           const uint32_t *ms, uint32_t nsites)
{
    if (!f || !np || !nsites || !mp || !ms) return LMB_E_ARG;
    std::string grp;
    {
        std::lock_guard<std::mutex> lk(f->mu);
        Node *g = replicate(f, rep);
        if (g->children.count("MaxParticleCounts") || g->children.count("MaxSiteCounts")) return LMB_E_STATE;
        grp = "Simulations/" + num(rep, 7);
    }
    // makeNewDataset (SimulationFile.cpp:2368-2393): chunks of min(16, n), gzip.
    int rc = chunked_dataset(f, grp, "MaxParticleCounts", Type::U32, {np}, {std::min<uint64_t>(FRAME_CHUNK, np)},
                             FRAME_GZIP, (const uint8_t *)mp);
    if (rc != LMB_OK) return rc;
    return chunked_dataset(f, grp, "MaxSiteCounts", Type::U32, {nsites},
                           {std::min<uint64_t>(FRAME_CHUNK, nsites)}, FRAME_GZIP, (const uint8_t *)ms);
}

static bool type_of(int code, Type *t)
{
    static const Type map[] = {Type::U8,  Type::I8,  Type::U16, Type::I16, Type::U32, Type::I32,
                               Type::U64, Type::I64, Type::F32, Type::F64, Type::STR};
    if (code < LMB_H5_U8 || code > LMB_H5_STRING) return false;
    *t = map[code - LMB_H5_U8];
    return true;
}

extern "C" int lmb_lmfile_create_group(lmb_lmfile *f, const char *path)
{
    if (!f || !path) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    return group_at(f->root, path) ? f->io_error : LMB_E_STATE;
}

extern "C" int lmb_lmfile_set_attribute(lmb_lmfile *f, const char *path, const char *name, int type, uint32_t rank,
                                        const uint64_t *dims, const void *data, uint32_t string_size)
{
    Type t;
    if (!f || !path || !name || !*name || !type_of(type, &t) || (rank && !dims) || rank > 32 ||
        (t == Type::STR && !string_size))
        return LMB_E_ARG;
    Attr a{name, t, t == Type::STR ? string_size : 0, std::vector<uint64_t>(dims, dims + rank), {}};
    size_t n = type_size(t, string_size);
    for (uint32_t i = 0; i < rank; i++) n *= dims[i];
    if (n && !data) return LMB_E_ARG;
    const uint8_t *b = (const uint8_t *)data;
    a.data.assign(b, b + n);
    if (!attr_fits(a)) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    // The object: a group (made if missing) or an existing dataset.
    const std::string p = path;
    const size_t slash = p.find_last_of('/');
    Node *parent = slash == std::string::npos ? &f->root : group_at(f->root, p.substr(0, slash));
    const std::string leaf = slash == std::string::npos ? p : p.substr(slash + 1);
    if (!parent) return LMB_E_STATE;
    Node *n0 = parent;
    if (!leaf.empty()) {
        auto it = parent->children.find(leaf);
        n0 = it != parent->children.end() && !it->second->group ? it->second.get() : group_at(*parent, leaf);
    }
    if (!n0) return LMB_E_STATE;
    set_attr(*n0, std::move(a));
    n0->dirty = true;
    return f->io_error;
}

extern "C" int lmb_lmfile_write_dataset(lmb_lmfile *f, const char *group, const char *name, int type, uint32_t rank,
                                        const uint64_t *dims, const uint64_t *chunk_dims, int gzip, int extendable,
                                        const void *data)
{
    Type t;
    if (!f || !group || !name || !*name || !type_of(type, &t) || t == Type::STR || !rank || !dims || rank > 32 ||
        gzip > 9 || (extendable && !chunk_dims))
        return LMB_E_ARG;
    const std::vector<uint64_t> d(dims, dims + rank);
    size_t n = type_size(t, 0);
    for (uint64_t x : d) n *= x;
    if (n && !data) return LMB_E_ARG;
    if (chunk_dims) {
        for (uint32_t i = 0; i < rank; i++)
            if (!chunk_dims[i] || (!(extendable && i == 0) && chunk_dims[i] > dims[i])) return LMB_E_ARG;
    }
    if (extendable) {
        std::lock_guard<std::mutex> lk(f->mu);
        Node *g = group_at(f->root, group);
        if (!g) return LMB_E_STATE;
        g->children.erase(name);
        std::vector<uint64_t> d0 = d;
        d0[0] = 0;
        Node *x = extendable_node(*g, name, t, d0, chunk_dims[0]);
        add_rows(*x, data, d[0]);
        x->chunk_dims.assign(chunk_dims, chunk_dims + rank);
        return f->io_error;
    }
    if (!chunk_dims || n == 0) {
        std::lock_guard<std::mutex> lk(f->mu);
        Node *g = group_at(f->root, group);
        if (!g) return LMB_E_STATE;
        contiguous(f, *g, name, t, d, data);
        return f->io_error;
    }
    return chunked_dataset(f, group, name, t, d, std::vector<uint64_t>(chunk_dims, chunk_dims + rank), gzip,
                           (const uint8_t *)data);
}

extern "C" int lmb_lmfile_flush(lmb_lmfile *f)
{
    if (!f) return LMB_E_ARG;
    int rc = drain(f);
    if (rc != LMB_OK) return rc;
    std::lock_guard<std::mutex> lk(f->mu);
    return commit(f);
}

extern "C" int lmb_lmfile_checkpoint(lmb_lmfile *f, char *out, uint64_t size)
{
    if (!f) return LMB_E_ARG;
    int rc = drain(f);
    if (rc != LMB_OK) return rc;
    const std::string chk = f->path + ".chk";
    {
        std::lock_guard<std::mutex> lk(f->mu);
        rc = commit(f);
        if (rc != LMB_OK) return rc;
        const int fd = open(chk.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (fd < 0) return LMB_E_IO;
        std::vector<uint8_t> buf(1 << 20);
        const uint64_t total = USER_BLOCK + f->eof;
        for (uint64_t off = 0; off < total && rc == LMB_OK;) {
            const size_t n = (size_t)std::min<uint64_t>(buf.size(), total - off);
            const ssize_t r = pread(f->fd, buf.data(), n, (off_t)off);
            if (r <= 0 || write(fd, buf.data(), (size_t)r) != r) rc = LMB_E_IO;
            off += r > 0 ? (uint64_t)r : 0;
        }
        if (close(fd) != 0) rc = LMB_E_IO;
        if (rc != LMB_OK) return rc;
    }
    if (out) {
        if (chk.size() + 1 > size) return LMB_E_ARG;
        memcpy(out, chk.c_str(), chk.size() + 1);
    }
    return LMB_OK;
}

extern "C" int lmb_lmfile_stats(lmb_lmfile *f, uint64_t *frames, uint64_t *chunk_bytes)
{
    if (!f) return LMB_E_ARG;
    std::lock_guard<std::mutex> lk(f->mu);
    if (frames) *frames = f->frames;
    if (chunk_bytes) *chunk_bytes = f->chunk_bytes;
    return LMB_OK;
}

extern "C" int lmb_lmfile_close(lmb_lmfile *f)
{
    if (!f) return LMB_E_ARG;
    const int rc = lmb_lmfile_flush(f);
    {
        std::lock_guard<std::mutex> lk(f->qmu);
        f->stop = true;
    }
    f->qcv.notify_all();
    if (f->writer.joinable()) f->writer.join();
    if (f->device >= 0) cudaSetDevice(f->device);
    for (auto &p : f->pinned) {
        if (p.host) cudaFreeHost(p.host);
        if (p.dev) cudaFree(p.dev);
        if (p.ready) cudaEventDestroy(p.ready);
        if (p.staged) cudaEventDestroy(p.staged);
    }
    if (f->copy) cudaStreamDestroy(f->copy);
    const int crc = close(f->fd) == 0 ? LMB_OK : LMB_E_IO;
    delete f;
    return rc != LMB_OK ? rc : crc;
}
