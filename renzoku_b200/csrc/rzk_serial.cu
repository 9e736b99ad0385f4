// rzk_serial.cu - warm restart of device scenes and the transport-matrix file format.
//
// Scene blobs: everything a built scene holds on the device (triangles, the reference-order
// BVH and its build products, the packed traversal records, the 4-wide nodes, the SAH
// any-hit tree, surfaces, materials, lights) plus its host-side counts, so that a serving
// process can restore a scene with host-to-device copies instead of rebuilding its trees.
// The arrays are listed once (scene_arrays) with their sizes derived from the counts, and
// serialise, size and restore all walk that one list.  No reference counterpart: the
// reference rebuilds its BVH from the scene file every run (aggregate_bvh.cc:48-240).
//
// Matrix files: MatrixC<Rgb>::save (matrix_c.cc:6-23) - the text header "rows cols\n",
// then the RGB floats of every entry, column by column - which is byte for byte the
// device layout [cols][rows][3] that rzk_gather_matrix writes.
#include "rzk_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace rzk {
namespace {

constexpr char kMagic[8] = {'R', 'Z', 'K', 'S', 'C', 'N', '0', '1'};

struct Array {
    void **ptr;
    size_t bytes;       // logical bytes (0 when the scene does not hold the array)
    size_t used = ~(size_t)0;   // bytes the build writes (the rest is spare capacity)
};

// The device arrays of a scene, in blob order.  Sizes follow the allocations of
// rzk_scene_create, bvh_build, build_sah_tree and setup_lights.
std::vector<Array> scene_arrays(rzk_scene *s) {
    const size_t n = (size_t)s->n_tris, cap = 2 * n, nl = (size_t)s->n_lights;
    const bool tree = s->n_tris > 0;
    auto f = [](size_t k) { return sizeof(float) * k; };
    auto i4 = [](size_t k) { return sizeof(int) * k; };
    auto v4 = [](size_t k) { return sizeof(float4) * k; };
    const size_t nn = (size_t)s->n_nodes;   // <= cap: the node arrays keep one spare entry
    std::vector<Array> a = {
        {(void **)&s->d_v, f(9 * n)},
        {(void **)&s->d_tp, f(3 * n)},
        {(void **)&s->d_tri_surf, i4(n)},
        {(void **)&s->d_surf, sizeof(int4) * (size_t)std::max(s->n_surfs, 1)},
        {(void **)&s->d_mats, sizeof(rzk_material) * (size_t)s->n_mats},
        {(void **)&s->d_tri_n, tree ? f(3 * n) : 0},
        {(void **)&s->d_tri_u, tree ? f(3 * n) : 0},
        {(void **)&s->d_tri_area, tree ? f(n) : 0},
        {(void **)&s->d_bmin, tree ? f(3 * n) : 0},
        {(void **)&s->d_bmax, tree ? f(3 * n) : 0},
        {(void **)&s->d_codes, tree ? i4(n) : 0},
        {(void **)&s->d_sorted_codes, tree ? i4(n) : 0},
        {(void **)&s->d_perm, tree ? i4(n) : 0},
        {(void **)&s->d_start, tree ? i4(cap) : 0, i4(nn)},
        {(void **)&s->d_end, tree ? i4(cap) : 0, i4(nn)},
        {(void **)&s->d_left, tree ? i4(cap) : 0, i4(nn)},
        {(void **)&s->d_right, tree ? i4(cap) : 0, i4(nn)},
        {(void **)&s->d_level, tree ? i4(cap) : 0, i4(nn)},
        {(void **)&s->d_nbmin, tree ? f(3 * cap) : 0, f(3 * nn)},
        {(void **)&s->d_nbmax, tree ? f(3 * cap) : 0, f(3 * nn)},
        {(void **)&s->d_nodes, tree ? v4(2 * (cap + 1)) : 0, v4(2 * (nn + 1))},
        {(void **)&s->d_tri_isect, tree ? v4(3 * n) : 0},
        {(void **)&s->d_tri_shade, tree ? v4(2 * n) : 0},
        {(void **)&s->d_wide, s->d_wide ? v4(8 * (size_t)std::max(1, s->n_wide)) : 0, v4(8 * (size_t)s->n_wide)},
        {(void **)&s->d_trav, s->d_trav ? s->trav_bytes : 0},
        {(void **)&s->d_lights, sizeof(DevLight) * nl},
        {(void **)&s->d_light_pdf, f(nl)},
        {(void **)&s->d_light_cdf, f(nl)},
    };
    return a;
}

// host-side state, fixed-size part
struct Header {
    char magic[8];
    uint32_t version, n_arrays;
    int32_t n_tris, n_nodes, n_levels, n_surfs, n_mats, n_lights, n_wide, trav_depth, build_trav, pad;
    float tmin, box[6], pad2;
    uint64_t trav_bytes, n_level_first, n_level_last, n_light_surf;
};

struct Writer {
    char *p;
    size_t cap, off = 0;
    bool ok = true;
    void put(const void *src, size_t b) {
        if (p) {
            if (off + b > cap) { ok = false; return; }
            if (b) std::memcpy(p + off, src, b);
        }
        off += b;
    }
};

struct Reader {
    const char *p;
    size_t size, off = 0;
    bool get(void *dst, size_t b) {
        if (b > size - off) return false;
        if (b) std::memcpy(dst, p + off, b);
        off += b;
        return true;
    }
};

// writes (or, with w.p == nullptr, measures) a scene's blob; device arrays are copied
// into the buffer only when `copy` is set
rzk_status write_scene(rzk_scene *s, Writer &w, cudaStream_t st, bool copy) {
    Header h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kMagic, 8);
    std::vector<Array> arrays = scene_arrays(s);
    h.version = 1;
    h.n_arrays = (uint32_t)arrays.size();
    h.n_tris = s->n_tris; h.n_nodes = s->n_nodes; h.n_levels = s->n_levels; h.n_surfs = s->n_surfs;
    h.n_mats = s->n_mats; h.n_lights = s->n_lights; h.n_wide = s->n_wide; h.trav_depth = s->trav_depth;
    h.build_trav = s->build_trav ? 1 : 0;
    h.tmin = s->tmin;
    for (int i = 0; i < 6; ++i) h.box[i] = s->box[i];
    h.trav_bytes = s->trav_bytes;
    h.n_level_first = s->level_first.size();
    h.n_level_last = s->level_last.size();
    h.n_light_surf = s->light_surf.size();
    w.put(&h, sizeof(h));
    w.put(s->level_first.data(), sizeof(int) * s->level_first.size());
    w.put(s->level_last.data(), sizeof(int) * s->level_last.size());
    w.put(s->light_surf.data(), sizeof(int) * s->light_surf.size());
    for (const Array &a : arrays) {
        const uint64_t b = *a.ptr ? a.bytes : 0;
        w.put(&b, sizeof(b));
        if (w.p && copy && b) {
            if (w.off + b > w.cap) { w.ok = false; return RZK_ERR_CAPACITY; }
            // the spare capacity was never written: zeros keep the blob deterministic
            const size_t u = std::min<size_t>(b, a.used);
            RZK_CUDA_TRY(cudaMemcpyAsync(w.p + w.off, *a.ptr, u, cudaMemcpyDeviceToHost, st));
            if (u < b) std::memset(w.p + w.off + u, 0, b - u);
        }
        w.off += b;
    }
    if (!w.ok) return RZK_ERR_CAPACITY;
    return RZK_OK;
}

void free_arrays(rzk_scene *s) {
    for (const Array &a : scene_arrays(s))
        if (*a.ptr) { cudaFree(*a.ptr); *a.ptr = nullptr; }
}

}  // namespace
}  // namespace rzk

using namespace rzk;

extern "C" {

rzk_status rzk_scene_serialized_size(rzk_scene *scene, size_t *bytes) {
    if (!scene || !bytes) return RZK_ERR_INVALID;
    Writer w{nullptr, 0};
    rzk_status r = write_scene(scene, w, nullptr, false);
    if (r != RZK_OK) return r;
    *bytes = w.off;
    return RZK_OK;
}

rzk_status rzk_scene_serialize(rzk_scene *scene, void *h_buf, size_t cap, size_t *written, void *stream) {
    if (!scene || !h_buf || !written) return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    size_t need = 0;
    RZK_TRY(rzk_scene_serialized_size(scene, &need));
    if (need > cap) return RZK_ERR_CAPACITY;
    Writer w{(char *)h_buf, cap};
    RZK_TRY(write_scene(scene, w, st, true));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    *written = w.off;
    return RZK_OK;
}

rzk_status rzk_scene_deserialize(rzk_context *ctx, const void *h_buf, size_t size, void *stream, rzk_scene **out) {
    if (!ctx || !h_buf || !out) return RZK_ERR_INVALID;
    *out = nullptr;
    Reader rd{(const char *)h_buf, size};
    Header h;
    if (!rd.get(&h, sizeof(h)) || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1) return RZK_ERR_INVALID;
    if (h.n_tris < 0 || h.n_nodes < 0 || h.n_levels < 0 || h.n_surfs < 0 || h.n_mats < 0 || h.n_lights < 0 ||
        h.n_wide < 0 || h.n_level_first > (1u << 20) || h.n_level_last > (1u << 20) ||
        h.n_light_surf > (uint64_t)h.n_lights)
        return RZK_ERR_INVALID;
    rzk_scene *s = new rzk_scene();
    auto fail = [&](rzk_status e) {
        free_arrays(s);
        delete s;
        return e;
    };
    s->ctx = ctx;
    s->n_tris = h.n_tris; s->n_nodes = h.n_nodes; s->n_levels = h.n_levels; s->n_surfs = h.n_surfs;
    s->n_mats = h.n_mats; s->n_lights = h.n_lights; s->n_wide = h.n_wide; s->n_wide_cap = h.n_wide;
    s->trav_depth = h.trav_depth; s->build_trav = h.build_trav != 0; s->tmin = h.tmin;
    for (int i = 0; i < 6; ++i) s->box[i] = h.box[i];
    s->trav_bytes = (size_t)h.trav_bytes;
    s->level_first.resize(h.n_level_first);
    s->level_last.resize(h.n_level_last);
    s->light_surf.resize(h.n_light_surf);
    if (!rd.get(s->level_first.data(), sizeof(int) * s->level_first.size()) ||
        !rd.get(s->level_last.data(), sizeof(int) * s->level_last.size()) ||
        !rd.get(s->light_surf.data(), sizeof(int) * s->light_surf.size()))
        return fail(RZK_ERR_INVALID);
    // every array's recorded size must be 0 or the size its counts give
    std::vector<Array> arrays = scene_arrays(s);
    // d_wide and d_trav are sized by the blob (held only when the source scene built them)
    std::vector<uint64_t> sizes(arrays.size());
    std::vector<size_t> offs(arrays.size());
    for (size_t k = 0; k < arrays.size(); ++k) {
        if (!rd.get(&sizes[k], sizeof(uint64_t))) return fail(RZK_ERR_INVALID);
        offs[k] = rd.off;
        if (sizes[k] > size - rd.off) return fail(RZK_ERR_INVALID);
        rd.off += (size_t)sizes[k];
    }
    if (h.n_arrays != arrays.size() || rd.off != size) return fail(RZK_ERR_INVALID);
    for (size_t k = 0; k < arrays.size(); ++k)   // no any-hit tree in the blob: none here either
        if (arrays[k].ptr == (void **)&s->d_trav && sizes[k] == 0) s->trav_bytes = 0;
    const size_t wide_bytes = sizeof(float4) * 8 * (size_t)std::max(1, h.n_wide);
    for (size_t k = 0; k < arrays.size(); ++k) {
        const bool is_wide = arrays[k].ptr == (void **)&s->d_wide, is_trav = arrays[k].ptr == (void **)&s->d_trav;
        const size_t expect = is_wide ? wide_bytes : (is_trav ? s->trav_bytes : arrays[k].bytes);
        if (sizes[k] != 0 && sizes[k] != expect) return fail(RZK_ERR_INVALID);
        if (sizes[k] == 0 && expect != 0 && !is_wide && !is_trav) return fail(RZK_ERR_INVALID);
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "scene restore", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    const char *base = (const char *)h_buf;
    for (size_t k = 0; k < arrays.size(); ++k) {
        if (sizes[k] == 0) continue;
        // the surfaces and materials were always allocated (16 bytes when empty)
        e = cudaMalloc(arrays[k].ptr, std::max<size_t>((size_t)sizes[k], 16));
        if (e != cudaSuccess) {
            set_last_cuda_error(e, "scene restore", __FILE__, __LINE__);
            return fail(RZK_ERR_NOMEM);
        }
        s->device_bytes += (size_t)sizes[k];
        e = cudaMemcpyAsync(*arrays[k].ptr, base + offs[k], (size_t)sizes[k], cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            set_last_cuda_error(e, "scene restore", __FILE__, __LINE__);
            return fail(RZK_ERR_CUDA);
        }
    }
    if (!s->d_mats) {   // n_mats == 0: rzk_scene_create holds a 16-byte stand-in
        e = cudaMalloc((void **)&s->d_mats, 16);
        if (e != cudaSuccess) return fail(RZK_ERR_NOMEM);
    }
    for (void **p : {(void **)&s->d_v, (void **)&s->d_tp, (void **)&s->d_tri_surf})
        if (!*p && (e = cudaMalloc(p, 16)) != cudaSuccess) return fail(RZK_ERR_NOMEM);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        set_last_cuda_error(e, "scene restore", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    *out = s;
    return RZK_OK;
}

rzk_status rzk_matrix_save(const char *path, const float *d_matrix, int rows, int cols, void *stream) {
    if (!path || rows < 0 || cols < 0 || ((size_t)rows * cols > 0 && !d_matrix)) return RZK_ERR_INVALID;
    const size_t n = 3 * (size_t)rows * cols;
    std::vector<float> h(n);
    cudaStream_t st = (cudaStream_t)stream;
    if (n) {
        RZK_CUDA_TRY(cudaMemcpyAsync(h.data(), d_matrix, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaStreamSynchronize(st));
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return RZK_ERR_INVALID;
    const bool ok = std::fprintf(f, "%d %d\n", rows, cols) > 0 && std::fwrite(h.data(), sizeof(float), n, f) == n;
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? RZK_OK : RZK_ERR_INVALID;
}

// Reads the header line "rows cols\n" exactly (MatrixC::load's fscanf("%d %d\n") would also
// swallow data bytes that look like white space, matrix_c.cc:32).
static bool read_matrix_header(FILE *f, int *rows, int *cols) {
    char line[64];
    int k = 0, c;
    while ((c = std::fgetc(f)) != EOF && c != '\n' && k < 63) line[k++] = (char)c;
    if (c != '\n') return false;
    line[k] = 0;
    return std::sscanf(line, "%d %d", rows, cols) == 2 && *rows >= 0 && *cols >= 0;
}

rzk_status rzk_matrix_file_info(const char *path, int *rows, int *cols) {
    if (!path || !rows || !cols) return RZK_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return RZK_ERR_INVALID;
    const bool ok = read_matrix_header(f, rows, cols);
    std::fclose(f);
    return ok ? RZK_OK : RZK_ERR_INVALID;
}

rzk_status rzk_matrix_load(const char *path, float *d_matrix, int rows, int cols, void *stream) {
    if (!path || rows < 0 || cols < 0 || ((size_t)rows * cols > 0 && !d_matrix)) return RZK_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return RZK_ERR_INVALID;
    int r = 0, c = 0;
    if (!read_matrix_header(f, &r, &c) || r != rows || c != cols) {
        std::fclose(f);
        return RZK_ERR_INVALID;
    }
    const size_t n = 3 * (size_t)rows * cols;
    std::vector<float> h(n);
    const bool ok = std::fread(h.data(), sizeof(float), n, f) == n;
    std::fclose(f);
    if (!ok) return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (n) {
        RZK_CUDA_TRY(cudaMemcpyAsync(d_matrix, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
        RZK_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return RZK_OK;
}

}  // extern "C"
