// extern "C" boundary of libvision_b200.so (declared in include/vision_b200.h).
#include "../../include/vision_b200.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "vs_host.h"
#include "vs_launch.h"
#include "vs_microfacet.h"
#include "vs_cache_render.h"
#include "vs_mlp.h"
#include "vs_server.h"
#include "vs_wavefront.h"

using namespace vs;

struct vs_context {
    int device = -1;
    cudaStream_t stream = nullptr;
    mutable std::mutex mu;
    std::string error;
    bool consts_uploaded = false;
};

namespace {

template <typename T>
struct DevBuf {
    T *ptr = nullptr;
    size_t count = 0;
    cudaError_t upload(const std::vector<T> &v) {
        free();
        if (v.empty()) return cudaSuccess;
        cudaError_t e = cudaMalloc(&ptr, v.size() * sizeof(T));
        if (e != cudaSuccess) { ptr = nullptr; return e; }
        count = v.size();
        return cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    }
    cudaError_t alloc(size_t n) {
        if (n <= count && ptr) return cudaSuccess;
        free();
        cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e != cudaSuccess) { ptr = nullptr; return e; }
        count = n;
        return cudaSuccess;
    }
    void free() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
};

}  // namespace

struct vs_scene {
    vs_context *ctx = nullptr;
    std::mutex mu;
    HostScene host;
    bool built = false;
    bool uploaded = false;
    DevBuf<Bvh8Node> nodes;
    DevBuf<float> tri_v;
    DevBuf<float4> vtx;
    DevBuf<uint4> prims;
    DevBuf<Instance> instances;
    DevBuf<Material> materials;
    DevBuf<AreaLight> lights;
    DevBuf<AliasEntry> prim_alias, light_alias;
    DevBuf<float> prim_pmf, light_pmf, spd, luts;
    DevBuf<float> env_tex, env_marginal_func, env_cond_func, rgb2spec;
    DevBuf<float> tex_texels;
    DevBuf<TextureRec> textures;
    DevBuf<AliasEntry> env_marginal, env_cond, filter_alias;
    DevBuf<float> filter_tab;
    // Two-level scenes: top-level leaf entries and per-instance transforms.
    DevBuf<uint32_t> tlas_inst;
    DevBuf<float4> inst_xf;
    // Film and per-sample radiance (scratch between the megakernel and the film pass).
    DevBuf<float4> film32, exposed;
    DevBuf<double> film64;
    DevBuf<float4> radiance;
    // Path counter of the persistent (regenerating) megakernel.
    DevBuf<unsigned long long> path_counter;
    int schedule = VS_SCHEDULE_WAVEFRONT;
    // Path slots of the wavefront schedule.
    struct WfBufs {
        DevBuf<float4> o, d, tp, lam, pdf, L, sh_o, sh_d, sh_c;
        DevBuf<uint4> st;
        DevBuf<Hit> hit;
        DevBuf<uint32_t> q0, q1, tq, count;
        DevBuf<uint32_t> bin_key, bins, binned, sh_perm;  // ray binning (VS_SCHEDULE_WAVEFRONT_BINNED)
        uint32_t capacity = 0;
        bool binning = false;
        void free() {
            o.free(); d.free(); tp.free(); lam.free(); pdf.free(); L.free(); sh_o.free(); sh_d.free(); sh_c.free();
            st.free(); hit.free(); q0.free(); q1.free(); tq.free(); count.free();
            bin_key.free(); bins.free(); binned.free(); sh_perm.free();
            capacity = 0;
            binning = false;
        }
        cudaError_t ensure(uint32_t n, bool with_bins) {
            if (n <= capacity && (binning || !with_bins)) return cudaSuccess;
            n = std::max(n, capacity);
            free();
            cudaError_t e = cudaSuccess;
            for (DevBuf<float4> *b : {&o, &d, &tp, &lam, &pdf, &L, &sh_o, &sh_d, &sh_c})
                if (e == cudaSuccess) e = b->alloc(n);
            if (e == cudaSuccess) e = st.alloc(n);
            if (e == cudaSuccess) e = hit.alloc(n);
            if (e == cudaSuccess) e = q0.alloc(n);
            if (e == cudaSuccess) e = q1.alloc(n);
            if (e == cudaSuccess) e = tq.alloc(static_cast<size_t>(n) * kWfClasses);
            if (e == cudaSuccess) e = count.alloc(kWfCounters);
            if (with_bins) {
                if (e == cudaSuccess) e = bin_key.alloc(n);
                if (e == cudaSuccess) e = binned.alloc(n);
                if (e == cudaSuccess) e = sh_perm.alloc(n);
                if (e == cudaSuccess) e = bins.alloc(2 * kWfBins);
                // The sizes half must start at zero; k_bin_scan clears it after each use.
                if (e == cudaSuccess) e = cudaMemset(bins.ptr, 0, 2 * kWfBins * sizeof(uint32_t));
                // Valid slot and entry indices from the start.
                if (e == cudaSuccess) e = cudaMemset(binned.ptr, 0, static_cast<size_t>(n) * sizeof(uint32_t));
                if (e == cudaSuccess) e = cudaMemset(sh_perm.ptr, 0, static_cast<size_t>(n) * sizeof(uint32_t));
            }
            if (e != cudaSuccess) {
                free();
                return e;
            }
            capacity = n;
            binning = with_bins;
            return cudaSuccess;
        }
        WfBuffers view() const {
            WfBuffers b{};
            b.capacity = capacity;
            b.o = o.ptr; b.d = d.ptr; b.tp = tp.ptr; b.lam = lam.ptr; b.pdf = pdf.ptr; b.L = L.ptr;
            b.st = st.ptr; b.hit = hit.ptr; b.queue[0] = q0.ptr; b.queue[1] = q1.ptr;
            b.sh_o = sh_o.ptr; b.sh_d = sh_d.ptr; b.sh_c = sh_c.ptr; b.tq = tq.ptr; b.count = count.ptr;
            return b;
        }
        // The view with the ray-binning buffers (all four or none).
        WfBuffers view_binned() const {
            WfBuffers b = view();
            if (binning) {
                b.bin_key = bin_key.ptr;
                b.bins = bins.ptr;
                b.binned = binned.ptr;
                b.sh_perm = sh_perm.ptr;
            }
            return b;
        }
    } wf;
    // Cache-terminated rendering: per-pixel queries, training samples, the
    // material albedo/roughness table of the feature encoding.
    struct CacheBufs {
        DevBuf<uint16_t> q_feat, t_feat, b_feat;
        DevBuf<CacheQueryRec> q_rec;
        DevBuf<CacheTrainRec> t_rec;
        DevBuf<float4> q_out, b_out, targets, mat;
        DevBuf<uint32_t> suffix_list, suffix_count;  // training paths of a wavefront frame
        uint32_t npix = 0, n_train = 0;  // sizes of the last frame (0: none rendered)
        void free() {
            q_feat.free(); t_feat.free(); b_feat.free(); q_rec.free(); t_rec.free();
            q_out.free(); b_out.free(); targets.free(); mat.free(); suffix_list.free(); suffix_count.free();
            npix = n_train = 0;
        }
    } cachebuf;
    uint32_t film_frames = 0;
    bool film64_valid = false;
    bool film64sq_valid = false;  // the second half of film64 holds sums of squares
    // Optional CUDA-event timing of the megakernel and film launches.
    bool timing = false;
    std::vector<cudaEvent_t> ev_render, ev_film;  // start/stop pairs
    cudaEvent_t ev_join = nullptr;
    // Real-time ReSTIR state: per-pixel buffers at the current resolution and
    // the previous frame's camera.
    struct Rt {
        DevBuf<RtSurface> surf[2];
        DevBuf<RtSurfaceExt> ext[2];
        DevBuf<RtHitBsdf> hit_bsdf;
        DevBuf<float2> motion;
        DevBuf<DiReservoir> di[2], di_pass;
        DevBuf<GiReservoir> gi[2], gi_pass, gi_init;
        DevBuf<float4> di_radiance, gi_radiance;
        DevBuf<float4> di_stage, di_ray;
        DevBuf<Hit> di_hit;
        DevBuf<uint32_t> di_list, di_count;
        DevBuf<float2> gs_nb;
        DevBuf<float4> gs_ray;
        DevBuf<uint8_t> gs_vis;
        DevBuf<uint32_t> gs_list, gs_count;
        uint32_t width = 0, height = 0;
        bool have_prev = false;
        Camera prev_cam{};
        m4 prev_w2c{};
        f3 prev_pos{};
        RtParams last{};
        bool rendered = false;
        void free() {
            for (int k = 0; k < 2; ++k) {
                surf[k].free(); ext[k].free(); di[k].free(); gi[k].free();
            }
            hit_bsdf.free(); motion.free(); di_pass.free(); gi_pass.free(); gi_init.free();
            di_radiance.free(); gi_radiance.free();
            di_stage.free(); di_ray.free(); di_hit.free(); di_list.free(); di_count.free();
            gs_nb.free(); gs_ray.free(); gs_vis.free(); gs_list.free(); gs_count.free();
        }
        RtBuffers view() const {
            RtBuffers b{};
            for (int k = 0; k < 2; ++k) {
                b.surf[k] = surf[k].ptr;
                b.ext[k] = ext[k].ptr;
                b.di[k] = di[k].ptr;
                b.gi[k] = gi[k].ptr;
            }
            b.hit_bsdf = hit_bsdf.ptr;
            b.motion = motion.ptr;
            b.di_pass = di_pass.ptr;
            b.gi_pass = gi_pass.ptr;
            b.gi_init = gi_init.ptr;
            b.di_radiance = di_radiance.ptr;
            b.gi_radiance = gi_radiance.ptr;
            b.di_stage = di_stage.ptr;
            b.di_ray = di_ray.ptr;
            b.di_hit = di_hit.ptr;
            b.di_list = di_list.ptr;
            b.di_count = di_count.ptr;
            b.gs_nb = gs_nb.ptr;
            b.gs_ray = gs_ray.ptr;
            b.gs_vis = gs_vis.ptr;
            b.gs_list = gs_list.ptr;
            b.gs_count = gs_count.ptr;
            return b;
        }
    } rt;

    // SVGF denoiser of the real-time frame: G-buffer and history by frame
    // parity, three rotating SVGFData buffers, the denoised frame.
    struct Svgf {
        DevBuf<SvgfGeom> geom[2];
        DevBuf<float> history[2];
        DevBuf<float2> motion;
        DevBuf<float4> albedo, emission, out;
        DevBuf<SvgfData> data[3];
        uint32_t width = 0, height = 0;
        uint32_t prev = 0;      // SVGFData buffer holding the previous frame's result
        bool on = false;        // vs_denoiser_enable
        bool rendered = false;  // a frame ran with the denoiser
        void free() {
            for (int k = 0; k < 2; ++k) {
                geom[k].free();
                history[k].free();
            }
            for (int k = 0; k < 3; ++k) data[k].free();
            motion.free(); albedo.free(); emission.free(); out.free();
            width = height = 0;
            rendered = false;
        }
        SvgfBuffers view(const float4 *radiance) const {
            SvgfBuffers b{};
            for (int k = 0; k < 2; ++k) {
                b.geom[k] = geom[k].ptr;
                b.history[k] = history[k].ptr;
            }
            for (int k = 0; k < 3; ++k) b.data[k] = data[k].ptr;
            b.motion = motion.ptr;
            b.albedo = albedo.ptr;
            b.emission = emission.ptr;
            b.radiance = radiance;
            b.out = out.ptr;
            return b;
        }
    } svgf;

    ~vs_scene() {
        for (cudaEvent_t e : ev_render) cudaEventDestroy(e);
        for (cudaEvent_t e : ev_film) cudaEventDestroy(e);
        if (ev_join) cudaEventDestroy(ev_join);
        nodes.free(); tri_v.free(); vtx.free(); prims.free(); instances.free(); materials.free(); lights.free();
        prim_alias.free(); light_alias.free(); prim_pmf.free(); light_pmf.free(); spd.free(); luts.free();
        env_tex.free(); env_marginal_func.free(); env_cond_func.free(); rgb2spec.free(); env_marginal.free(); env_cond.free();
        tex_texels.free(); textures.free();
        filter_tab.free(); filter_alias.free(); tlas_inst.free(); inst_xf.free();
        film32.free(); exposed.free(); film64.free(); radiance.free(); path_counter.free(); wf.free();
        rt.free();
        svgf.free();
        cachebuf.free();
    }

    // Device memory of the scene proper (geometry, BVH, materials, lights,
    // sampling tables, environment, filter and LUTs), not its film or render
    // scratch.
    uint64_t device_bytes() const {
        auto b = [](const auto &buf) { return static_cast<uint64_t>(buf.count) * sizeof(*buf.ptr); };
        return b(nodes) + b(tri_v) + b(vtx) + b(prims) + b(instances) + b(materials) + b(lights) + b(prim_alias) +
               b(light_alias) + b(prim_pmf) + b(light_pmf) + b(spd) + b(luts) + b(env_tex) + b(env_marginal_func) +
               b(env_cond_func) + b(rgb2spec) + b(env_marginal) + b(env_cond) + b(filter_tab) + b(filter_alias) +
               b(tex_texels) + b(textures) +
               b(tlas_inst) + b(inst_xf);
    }

    // Device memory of the per-pixel buffers a real-time frame keeps resident:
    // reservoirs, surfaces and the other ReSTIR buffers, the film and, on the
    // wavefront schedule, the path slots.
    uint64_t rt_resident_bytes() const {
        auto b = [](const auto &buf) { return static_cast<uint64_t>(buf.count) * sizeof(*buf.ptr); };
        uint64_t n = b(film32) + b(exposed) + b(radiance);
        for (int k = 0; k < 2; ++k) n += b(rt.surf[k]) + b(rt.ext[k]) + b(rt.di[k]) + b(rt.gi[k]);
        n += b(rt.hit_bsdf) + b(rt.motion) + b(rt.di_pass) + b(rt.gi_pass) + b(rt.gi_init) + b(rt.di_radiance) +
             b(rt.gi_radiance) + b(rt.di_stage) + b(rt.di_ray) + b(rt.di_hit) + b(rt.di_list) + b(rt.di_count) +
             b(rt.gs_nb) + b(rt.gs_ray) + b(rt.gs_vis) + b(rt.gs_list) + b(rt.gs_count);
        for (int k = 0; k < 2; ++k) n += b(svgf.geom[k]) + b(svgf.history[k]);
        for (int k = 0; k < 3; ++k) n += b(svgf.data[k]);
        n += b(svgf.motion) + b(svgf.albedo) + b(svgf.emission) + b(svgf.out);
        n += b(wf.o) + b(wf.d) + b(wf.tp) + b(wf.lam) + b(wf.pdf) + b(wf.L) + b(wf.sh_o) + b(wf.sh_d) + b(wf.sh_c) +
             b(wf.st) + b(wf.hit) + b(wf.q0) + b(wf.q1) + b(wf.tq) + b(wf.count) + b(wf.bin_key) + b(wf.bins) +
             b(wf.binned) + b(wf.sh_perm);
        return n;
    }

    DeviceScene device_view() const {
        DeviceScene d{};
        d.nodes = reinterpret_cast<const uint4 *>(nodes.ptr);
        d.tri_v = reinterpret_cast<const float4 *>(tri_v.ptr);
        d.vtx = vtx.ptr;
        d.prims = prims.ptr;
        d.instances = instances.ptr;
        d.materials = materials.ptr;
        d.lights = lights.ptr;
        d.prim_alias = prim_alias.ptr;
        d.prim_pmf = prim_pmf.ptr;
        d.light_alias = light_alias.ptr;
        d.light_pmf = light_pmf.ptr;
        d.spd = spd.ptr;
        d.luts = luts.ptr;
        d.has_env = host.has_env ? 1u : 0u;
        d.env = host.env;
        d.env_index = host.ip.light_count - 1u;
        d.env_tex = reinterpret_cast<const float4 *>(env_tex.ptr);
        d.env_marginal = env_marginal.ptr;
        d.env_marginal_func = env_marginal_func.ptr;
        d.env_cond = env_cond.ptr;
        d.env_cond_func = env_cond_func.ptr;
        d.rgb2spec = reinterpret_cast<const float4 *>(rgb2spec.ptr);
        d.tex_texels = reinterpret_cast<const float4 *>(tex_texels.ptr);
        d.textures = reinterpret_cast<const uint4 *>(textures.ptr);
        d.filter_tab = filter_tab.ptr;
        d.filter_alias = filter_alias.ptr;
        d.filter_integral = host.filter_integral;
        d.cam = host.cam;
        d.ip = host.ip;
        d.node_count = static_cast<uint32_t>(host.nodes.size());
        d.prim_count = static_cast<uint32_t>(host.prim_inst.size());
        d.two_level = host.two_level ? 1u : 0u;
        d.tlas_inst = tlas_inst.ptr;
        d.inst_xf = inst_xf.ptr;
        d.stats = nullptr;
        return d;
    }
};

namespace {

// Upper bound on paths per megakernel launch; sizes the radiance scratch
// (16 bytes per path).
constexpr uint64_t kMaxPathsPerLaunch = 1ull << 26;
// Path slots of one wavefront wave (208 B each: 832 MiB).
constexpr uint64_t kWfWaveSlots = 1ull << 22;

int fail(const vs_context *ctx, int code, const std::string &msg) {
    if (ctx) {
        std::lock_guard<std::mutex> lock(ctx->mu);
        const_cast<vs_context *>(ctx)->error = msg;
    }
    return code;
}

int cuda_fail(const vs_context *ctx, cudaError_t e, const char *where) {
    return fail(ctx, VS_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define VS_CUDA(call, where)                                        \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where);    \
    } while (0)

cudaStream_t pick_stream(const vs_scene *s, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : s->ctx->stream;
}

// Shading classes of the wavefront that a scene can produce: misses and one
// class per material type present.
// Mix / add materials have a shading class of their own (a composite BSDF of
// two child lobe sets), compiled only into the wavefront schedule's class
// kernels; the kernels built for a fixed material set (megakernel schedules,
// the allocation-free render, the instrumented render, the radiance-cache
// frame, the render server) do not take them.
bool has_mix(const HostScene &h) {
    for (const Material &mt : h.materials)
        if (mt.type == kMatMix) return true;
    return false;
}

uint32_t shading_classes(const HostScene &h) {
    uint32_t m = 1u;
    for (const Material &mt : h.materials) m |= 1u << (1u + mt.type);
    return m;
}

// Per instance: the world-to-object rows and (mesh root node, first
// primitive) as bits (DeviceScene::inst_xf).
std::vector<float4> instance_transforms(const HostScene &h) {
    std::vector<float4> x(4 * h.instances.size());
    for (size_t i = 0; i < h.instances.size(); ++i) {
        const m4 &m = h.inst_w2o[i];
        for (int r = 0; r < 3; ++r) x[4 * i + r] = make_float4(m.m[0][r], m.m[1][r], m.m[2][r], m.m[3][r]);
        x[4 * i + 3] = make_float4(bits_float(h.blas_root[h.inst_mesh[i]]), bits_float(h.instances[i].first_prim),
                                   bits_float(h.inst_mesh[i]), 0.0f);
    }
    return x;
}

int upload_scene(vs_scene *s) {
    vs_context *ctx = s->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!ctx->consts_uploaded) {
        const Cie5 &c = cie5();
        VS_CUDA(upload_spectral_consts(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(rt_all::upload_spectral_consts_rt(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(rt_diffuse::upload_spectral_consts_rt(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(upload_spectral_consts_serve(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(upload_spectral_consts_cache(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(upload_spectral_consts_wf(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        VS_CUDA(upload_spectral_consts_svgf(c.x, c.y, c.z, c.d65, c.y_integral), "spectral constants");
        ctx->consts_uploaded = true;
    }
    const HostScene &h = s->host;
    std::vector<float4> vtx(h.pos.size() * 2);
    for (size_t i = 0; i < h.pos.size(); ++i) {
        vtx[2 * i] = make_float4(h.pos[i].x, h.pos[i].y, h.pos[i].z, h.uv[i].x);
        vtx[2 * i + 1] = make_float4(h.nrm[i].x, h.nrm[i].y, h.nrm[i].z, h.uv[i].y);
    }
    std::vector<uint4> prims(h.prim_inst.size());
    for (size_t i = 0; i < prims.size(); ++i)
        prims[i] = make_uint4(h.idx[3 * i], h.idx[3 * i + 1], h.idx[3 * i + 2], h.prim_inst[i]);
    VS_CUDA(s->nodes.upload(h.nodes), "upload nodes");
    VS_CUDA(s->tri_v.upload(h.tri_v), "upload triangles");
    VS_CUDA(s->vtx.upload(vtx), "upload vertices");
    VS_CUDA(s->prims.upload(prims), "upload primitives");
    VS_CUDA(s->instances.upload(h.instances), "upload instances");
    VS_CUDA(s->materials.upload(h.materials), "upload materials");
    VS_CUDA(s->lights.upload(h.lights), "upload lights");
    VS_CUDA(s->prim_alias.upload(h.prim_alias), "upload alias");
    VS_CUDA(s->prim_pmf.upload(h.prim_pmf), "upload pmf");
    VS_CUDA(s->light_alias.upload(h.light_alias), "upload light alias");
    VS_CUDA(s->light_pmf.upload(h.light_pmf), "upload light pmf");
    std::vector<float> spd = h.spd;
    if (spd.empty()) spd.push_back(0.0f);
    VS_CUDA(s->spd.upload(spd), "upload spd");
    std::vector<float> luts(1, 0.0f);
    if (h.needs_luts) {
        const float *t = microfacet_luts();
        luts.assign(t, t + kLutFloats);
        luts.insert(luts.end(), coat_lut(), coat_lut() + (kLutSheen - kLutCoat));
        luts.insert(luts.end(), sheen_ltc_lut(), sheen_ltc_lut() + (kLutDeviceFloats - kLutSheen));
    }
    VS_CUDA(s->luts.upload(luts), "upload luts");
    if (h.has_env) {
        VS_CUDA(s->env_tex.upload(h.env_tex), "upload env");
        VS_CUDA(s->env_marginal.upload(h.env_marginal), "upload env");
        VS_CUDA(s->env_marginal_func.upload(h.env_marginal_func), "upload env");
        VS_CUDA(s->env_cond.upload(h.env_cond), "upload env");
        VS_CUDA(s->env_cond_func.upload(h.env_cond_func), "upload env");
    }
    // The RGB -> spectrum table: the environment's texels and textured
    // colour slots decode through it on the device.
    if (h.has_env || (!h.textures.empty() && !h.ip.srgb)) {
        const float *t = rgb2spec_table("");
        std::vector<float> tab(t, t + static_cast<size_t>(3) * 64 * 64 * 64 * 4);
        VS_CUDA(s->rgb2spec.upload(tab), "upload rgb2spec");
    } else {
        s->rgb2spec.free();
    }
    if (!h.textures.empty()) {
        VS_CUDA(s->tex_texels.upload(h.tex_texels), "upload textures");
        VS_CUDA(s->textures.upload(h.textures), "upload textures");
    } else {
        s->tex_texels.free();
        s->textures.free();
    }
    if (!h.filter_tab.empty()) {
        VS_CUDA(s->filter_tab.upload(h.filter_tab), "upload filter table");
        VS_CUDA(s->filter_alias.upload(h.filter_alias), "upload filter table");
    }
    s->tlas_inst.free();
    s->inst_xf.free();
    if (h.two_level) {
        VS_CUDA(s->tlas_inst.upload(h.tlas_inst), "upload top level");
        VS_CUDA(s->inst_xf.upload(instance_transforms(h)), "upload instances");
    }
    s->uploaded = true;
    return VS_OK;
}

int ensure_film(vs_scene *s) {
    vs_context *ctx = s->ctx;
    size_t npix = static_cast<size_t>(s->host.cam.width) * s->host.cam.height;
    VS_CUDA(s->film32.alloc(npix), "film alloc");
    VS_CUDA(s->exposed.alloc(npix), "film alloc");
    return VS_OK;
}

}  // namespace

namespace vs {

std::mutex &noalloc_scene_mutex(vs_scene *s) { return s->mu; }

// The caller holds s->mu (noalloc_scene_mutex) for this call and for every
// launch that uses the returned view, so a concurrent vs_scene_build_accel
// cannot free the buffers the view points to.
int noalloc_prepare(vs_scene *s, void *stream, DeviceScene *view, cudaStream_t *st, int *device) {
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot render");
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede vs_render_noalloc");
    if (has_mix(s->host)) return fail(ctx, VS_E_UNSUPPORTED, "mix / add materials in the allocation-free render");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    *view = s->device_view();
    *st = pick_stream(s, stream);
    *device = ctx->device;
    return VS_OK;
}

int noalloc_fail(vs_scene *s, int code, const char *msg) { return fail(s->ctx, code, msg); }

}  // namespace vs

extern "C" {

int vs_version(void) { return 100; }

int vs_context_create(int device, vs_context **out) {
    if (!out) return VS_E_INVALID;
    *out = nullptr;
    vs_context *ctx = new vs_context();
    ctx->device = device;
    if (device >= 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device >= n) {
            delete ctx;
            return VS_E_NO_DEVICE;
        }
        if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return VS_E_CUDA;
        }
    }
    *out = ctx;
    return VS_OK;
}

void vs_context_destroy(vs_context *ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *vs_last_error(const vs_context *ctx) {
    if (!ctx) return "null context";
    return ctx->error.c_str();
}

int vs_scene_load_json(vs_context *ctx, const char *json, size_t len, const char *base_dir, const char *table_cache,
                       vs_scene **out) {
    if (!ctx || !json || !out) return fail(ctx, VS_E_INVALID, "null argument");
    *out = nullptr;
    vs_scene *s = new vs_scene();
    s->ctx = ctx;
    try {
        load_scene_json(std::string(json, len), base_dir ? base_dir : "", table_cache ? table_cache : "", s->host);
    } catch (const std::exception &e) {
        std::string m = e.what();
        delete s;
        if (m.rfind("unsupported", 0) == 0) return fail(ctx, VS_E_UNSUPPORTED, m);
        return fail(ctx, VS_E_PARSE, m);
    }
    *out = s;
    return VS_OK;
}

void vs_scene_destroy(vs_scene *s) {
    if (!s) return;
    if (s->ctx && s->ctx->device >= 0) cudaSetDevice(s->ctx->device);
    delete s;
}

int vs_scene_build_accel(vs_scene *s) {
    if (!s) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->host.prim_inst.empty()) return fail(ctx, VS_E_STATE, "build_accel: the scene has no geometry");
    if (s->host.ip.light_count == 0) return fail(ctx, VS_E_STATE, "build_accel: the scene has no lights");
    try {
        build_bvh8(s->host);
    } catch (const std::exception &e) {
        return fail(ctx, VS_E_RANGE, e.what());
    }
    s->built = true;
    if (ctx->device >= 0) {
        int rc = upload_scene(s);
        if (rc != VS_OK) return rc;
    }
    return VS_OK;
}

int vs_scene_add_instance(vs_scene *s, const vs_vertex *vertices, uint32_t vert_num, const uint32_t *triangles,
                          uint32_t tri_num, const float *mat4, const char *material, uint32_t *instance_id) {
    if (!s || (vert_num && !vertices) || (tri_num && !triangles)) return fail(s ? s->ctx : nullptr, VS_E_INVALID, "null argument");
    vs_context *ctx = s->ctx;
    if (tri_num == 0 || vert_num == 0) return fail(ctx, VS_E_INVALID, "add_instance: empty mesh");
    for (size_t i = 0; i < 3u * static_cast<size_t>(tri_num); ++i)
        if (triangles[i] >= vert_num) return fail(ctx, VS_E_INVALID, "add_instance: triangle index out of range");
    m4 o2w = m4_identity();
    if (mat4)
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) o2w.m[c][r] = mat4[4 * c + r];
    std::lock_guard<std::mutex> lock(s->mu);
    uint32_t id = 0;
    try {
        static_assert(sizeof(vs_vertex) == 40, "sdk::Vertex is 40 bytes");
        id = scene_add_instance(s->host, reinterpret_cast<const float *>(vertices), vert_num, triangles, tri_num, o2w,
                                material ? std::string(material) : std::string());
    } catch (const std::exception &e) {
        std::string m = e.what();
        if (m.rfind("unsupported", 0) == 0) return fail(ctx, VS_E_UNSUPPORTED, m);
        if (m.rfind("json", 0) == 0) return fail(ctx, VS_E_PARSE, m);
        return fail(ctx, VS_E_INVALID, m);
    }
    s->built = false;
    s->uploaded = false;
    s->film_frames = 0;
    s->film64_valid = false;
    s->film64sq_valid = false;
    if (instance_id) *instance_id = id;
    return VS_OK;
}

int vs_scene_clear_geometries(vs_scene *s) {
    if (!s) return VS_E_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    scene_clear_geometries(s->host);
    s->built = false;
    s->uploaded = false;
    s->film_frames = 0;
    s->film64_valid = false;
    s->film64sq_valid = false;
    return VS_OK;
}

int vs_scene_invalidate(vs_scene *s) {
    if (!s) return VS_E_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    s->film_frames = 0;
    s->film64_valid = false;
    s->film64sq_valid = false;
    return VS_OK;
}

int vs_set_resolution(vs_scene *s, uint32_t width, uint32_t height) {
    if (!s || width == 0 || height == 0) return fail(s ? s->ctx : nullptr, VS_E_INVALID, "bad resolution");
    std::lock_guard<std::mutex> lock(s->mu);
    update_camera(s->host, width, height);
    s->film_frames = 0;
    s->film64_valid = false;
    s->film64sq_valid = false;
    return VS_OK;
}

int vs_camera_set(vs_scene *s, const float *c2w16, float fov_y_deg) {
    if (!s || !c2w16) return VS_E_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) s->host.cam.c2w.m[c][r] = c2w16[4 * c + r];
    float fov = fov_y_deg < 15.0f ? 15.0f : (fov_y_deg > 120.0f ? 120.0f : fov_y_deg);
    s->host.cam.tan_half_fov = std::tan(fov * kPi / 180.0f * 0.5f);
    s->film_frames = 0;
    s->film64_valid = false;
    s->film64sq_valid = false;
    return VS_OK;
}

int vs_scene_info_get(const vs_scene *s, vs_scene_info *o) {
    if (!s || !o) return VS_E_INVALID;
    const HostScene &h = s->host;
    o->vertex_count = static_cast<uint32_t>(h.pos.size());
    o->prim_count = static_cast<uint32_t>(h.prim_inst.size());
    o->instance_count = static_cast<uint32_t>(h.instances.size());
    o->material_count = static_cast<uint32_t>(h.materials.size());
    o->light_count = static_cast<uint32_t>(h.lights.size());
    o->prim_alias_count = static_cast<uint32_t>(h.prim_alias.size());
    o->spd_floats = static_cast<uint32_t>(h.spd.size());
    o->bvh_node_count = static_cast<uint32_t>(h.nodes.size());
    o->bvh_depth = h.bvh_depth;
    o->width = h.cam.width;
    o->height = h.cam.height;
    o->spectrum_dim = h.ip.spectrum_dim;
    o->max_depth = h.ip.max_depth;
    o->accel_built = s->built ? 1u : 0u;
    o->two_level = h.two_level ? 1u : 0u;
    o->mesh_count = static_cast<uint32_t>(h.meshes.size());
    return VS_OK;
}

namespace {
struct ExportView {
    const void *ptr;
    size_t bytes;
};
ExportView export_view(const vs_scene *s, int what) {
    const HostScene &h = s->host;
    switch (what) {
        case VS_EXPORT_POS: return {h.pos.data(), h.pos.size() * sizeof(f3)};
        case VS_EXPORT_NRM: return {h.nrm.data(), h.nrm.size() * sizeof(f3)};
        case VS_EXPORT_UV: return {h.uv.data(), h.uv.size() * sizeof(f2)};
        case VS_EXPORT_IDX: return {h.idx.data(), h.idx.size() * 4};
        case VS_EXPORT_PRIM_INST: return {h.prim_inst.data(), h.prim_inst.size() * 4};
        case VS_EXPORT_INSTANCES: return {h.instances.data(), h.instances.size() * sizeof(Instance)};
        case VS_EXPORT_MATERIALS: return {h.materials.data(), h.materials.size() * sizeof(Material)};
        case VS_EXPORT_LIGHTS: return {h.lights.data(), h.lights.size() * sizeof(AreaLight)};
        case VS_EXPORT_PRIM_ALIAS: return {h.prim_alias.data(), h.prim_alias.size() * sizeof(AliasEntry)};
        case VS_EXPORT_PRIM_PMF: return {h.prim_pmf.data(), h.prim_pmf.size() * 4};
        case VS_EXPORT_LIGHT_ALIAS: return {h.light_alias.data(), h.light_alias.size() * sizeof(AliasEntry)};
        case VS_EXPORT_LIGHT_PMF: return {h.light_pmf.data(), h.light_pmf.size() * 4};
        case VS_EXPORT_CAMERA: return {&h.cam, sizeof(Camera)};
        case VS_EXPORT_INTEGRATOR: return {&h.ip, sizeof(IntegratorParams)};
        case VS_EXPORT_SPD: return {h.spd.data(), h.spd.size() * 4};
        case VS_EXPORT_MATERIAL_RGB: return {h.material_rgb.data(), h.material_rgb.size() * sizeof(f3)};
        case VS_EXPORT_LIGHT_RGB: return {h.light_rgb.data(), h.light_rgb.size() * sizeof(f3)};
        case VS_EXPORT_BVH_NODES: return {h.nodes.data(), h.nodes.size() * sizeof(Bvh8Node)};
        case VS_EXPORT_BVH_TRIS: return {h.tri_v.data(), h.tri_v.size() * 4};
        case VS_EXPORT_ENV: return h.has_env ? ExportView{&h.env, sizeof(EnvLight)} : ExportView{nullptr, 0};
        case VS_EXPORT_ENV_TEX: return {h.env_tex.data(), h.env_tex.size() * 4};
        case VS_EXPORT_ENV_MARGINAL: return {h.env_marginal.data(), h.env_marginal.size() * sizeof(AliasEntry)};
        case VS_EXPORT_ENV_MARGINAL_FUNC: return {h.env_marginal_func.data(), h.env_marginal_func.size() * 4};
        case VS_EXPORT_ENV_COND: return {h.env_cond.data(), h.env_cond.size() * sizeof(AliasEntry)};
        case VS_EXPORT_ENV_COND_FUNC: return {h.env_cond_func.data(), h.env_cond_func.size() * 4};
        case VS_EXPORT_RGB2SPEC: return {rgb2spec_table(""), static_cast<size_t>(3) * 64 * 64 * 64 * 16};
        case VS_EXPORT_MESH_POS: return {h.mesh_pos.data(), h.mesh_pos.size() * sizeof(f3)};
        case VS_EXPORT_MESH_IDX: return {h.mesh_idx.data(), h.mesh_idx.size() * 4};
        case VS_EXPORT_MESHES: return {h.meshes.data(), h.meshes.size() * sizeof(HostScene::MeshRec)};
        case VS_EXPORT_TEXELS: return {h.tex_texels.data(), h.tex_texels.size() * sizeof(float)};
        case VS_EXPORT_TEXTURES: return {h.textures.data(), h.textures.size() * sizeof(TextureRec)};
        case VS_EXPORT_INST_MESH: return {h.inst_mesh.data(), h.inst_mesh.size() * 4};
        case VS_EXPORT_INST_W2O: return {h.inst_w2o.data(), h.inst_w2o.size() * sizeof(m4)};
        case VS_EXPORT_LUTS: {
            if (!h.needs_luts) return {nullptr, 0};
            return {microfacet_luts(), static_cast<size_t>(kLutFloats) * 4};
        }
        default: return {nullptr, static_cast<size_t>(-1)};
    }
}
}  // namespace

int vs_scene_export_size(const vs_scene *s, int what, size_t *bytes) {
    if (!s || !bytes) return VS_E_INVALID;
    ExportView v = export_view(s, what);
    if (v.bytes == static_cast<size_t>(-1)) return fail(s->ctx, VS_E_INVALID, "unknown export id");
    *bytes = v.bytes;
    return VS_OK;
}

int vs_scene_export(const vs_scene *s, int what, void *dst, size_t bytes) {
    if (!s || (!dst && bytes)) return VS_E_INVALID;
    ExportView v = export_view(s, what);
    if (v.bytes == static_cast<size_t>(-1)) return fail(s->ctx, VS_E_INVALID, "unknown export id");
    if (bytes != v.bytes) return fail(s->ctx, VS_E_INVALID, "export size mismatch");
    if (bytes) std::memcpy(dst, v.ptr, bytes);
    return VS_OK;
}

int vs_render(vs_scene *s, uint32_t frame_begin, uint32_t frame_count, int film_precision, void *stream) {
    if (!s) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot render");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede vs_render");
    if (frame_begin != 0 && frame_begin != s->film_frames)
        return fail(ctx, VS_E_STATE, "frames must continue the film (frame_begin == frames rendered) or restart at 0");
    if (film_precision == VS_FILM_FP64 && frame_begin != 0 && !s->film64_valid)
        return fail(ctx, VS_E_STATE, "FP64 film must be enabled from frame 0");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    int rc = ensure_film(s);
    if (rc != VS_OK) return rc;
    cudaStream_t st = pick_stream(s, stream);
    uint64_t npix = static_cast<uint64_t>(s->host.cam.width) * s->host.cam.height;
    // Sums (double4 per pixel) followed by sums of squares (double4 per pixel).
    if (film_precision == VS_FILM_FP64) VS_CUDA(s->film64.alloc(npix * 8), "film64 alloc");
    uint64_t frames_per_chunk = kMaxPathsPerLaunch / npix;
    if (frames_per_chunk == 0) return fail(ctx, VS_E_RANGE, "resolution above the per-launch path limit");
    if (frames_per_chunk > frame_count) frames_per_chunk = frame_count;
    VS_CUDA(s->radiance.alloc(static_cast<size_t>(frames_per_chunk * npix)), "radiance alloc");
    if (s->schedule == VS_SCHEDULE_PERSISTENT) VS_CUDA(s->path_counter.alloc(1), "path counter alloc");
    const bool wavefront = s->schedule == VS_SCHEDULE_WAVEFRONT || s->schedule == VS_SCHEDULE_WAVEFRONT_BINNED;
    if (!wavefront && has_mix(s->host))
        return fail(ctx, VS_E_UNSUPPORTED, "mix / add materials render with the wavefront schedules only");
    if (wavefront)
        VS_CUDA(s->wf.ensure(static_cast<uint32_t>(std::min<uint64_t>(frames_per_chunk * npix, kWfWaveSlots)),
                             s->schedule == VS_SCHEDULE_WAVEFRONT_BINNED),
                "wavefront slots alloc");
    DeviceScene dv = s->device_view();
    auto timed_event = [&](std::vector<cudaEvent_t> &v) -> cudaError_t {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        v.push_back(e);
        return cudaEventRecord(e, st);
    };
    for (uint32_t f = 0; f < frame_count; f += static_cast<uint32_t>(frames_per_chunk)) {
        uint32_t fc = static_cast<uint32_t>(std::min<uint64_t>(frames_per_chunk, frame_count - f));
        if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
        if (wavefront) {
            unsigned n = 0;
            VS_CUDA(launch_render_wavefront(dv, frame_begin + f, fc, s->radiance.ptr,
                                            s->schedule == VS_SCHEDULE_WAVEFRONT_BINNED ? s->wf.view_binned()
                                                                                        : s->wf.view(),
                                            shading_classes(s->host), st, &n),
                    "wavefront render");
            add_launches(n);
        } else {
            VS_CUDA(launch_render(dv, frame_begin + f, fc, s->radiance.ptr, st,
                                  s->schedule == VS_SCHEDULE_PERSISTENT ? s->path_counter.ptr : nullptr),
                    "render launch");
        }
        if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
        if (s->timing) VS_CUDA(timed_event(s->ev_film), "timing event");
        VS_CUDA(launch_film(s->radiance.ptr, static_cast<uint32_t>(npix), frame_begin + f, fc, s->film32.ptr,
                            film_precision == VS_FILM_FP64 ? s->film64.ptr : nullptr, st,
                            film_precision == VS_FILM_FP64 ? s->film64.ptr + npix * 4 : nullptr),
                "film launch");
        if (s->timing) VS_CUDA(timed_event(s->ev_film), "timing event");
    }
    // Later calls on the context stream (film download) must see this work.
    if (st != ctx->stream) {
        if (!s->ev_join) VS_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming), "join event");
        VS_CUDA(cudaEventRecord(s->ev_join, st), "join record");
        VS_CUDA(cudaStreamWaitEvent(ctx->stream, s->ev_join, 0), "join wait");
    }
    s->film_frames = frame_begin + frame_count;
    s->film64_valid = film_precision == VS_FILM_FP64 && (frame_begin == 0 || s->film64_valid);
    s->film64sq_valid = film_precision == VS_FILM_FP64 && (frame_begin == 0 || s->film64sq_valid);
    return VS_OK;
}

int vs_render_schedule_set(vs_scene *s, int schedule) {
    if (!s) return VS_E_INVALID;
    if (schedule != VS_SCHEDULE_GRID && schedule != VS_SCHEDULE_PERSISTENT && schedule != VS_SCHEDULE_WAVEFRONT &&
        schedule != VS_SCHEDULE_WAVEFRONT_BINNED)
        return fail(s->ctx, VS_E_INVALID,
                    "schedule must be VS_SCHEDULE_GRID, _PERSISTENT, _WAVEFRONT or _WAVEFRONT_BINNED");
    std::lock_guard<std::mutex> lock(s->mu);
    s->schedule = schedule;
    return VS_OK;
}

int vs_synchronize(vs_scene *s) {
    if (!s) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return VS_OK;
    VS_CUDA(cudaStreamSynchronize(ctx->stream), "synchronize");
    return VS_OK;
}

int vs_film_download(vs_scene *s, void *dst, size_t bytes, int which) {
    if (!s || !dst) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context has no film");
    std::lock_guard<std::mutex> lock(s->mu);
    size_t npix = static_cast<size_t>(s->host.cam.width) * s->host.cam.height;
    if (s->film_frames == 0) return fail(ctx, VS_E_STATE, "nothing rendered");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    if (which == VS_FILM_LINEAR || which == VS_FILM_EXPOSED || which == VS_FILM_DISPLAY || which == VS_FILM_HDR) {
        if (bytes != npix * 16) return fail(ctx, VS_E_INVALID, "film size mismatch");
        const float4 *src = s->film32.ptr;
        if (which != VS_FILM_LINEAR) {
            const uint32_t passes = which == VS_FILM_EXPOSED ? 1u : 2u;
            VS_CUDA(launch_picture(s->film32.ptr, static_cast<uint32_t>(npix), s->host.cam.exposure, s->host.tone_mapper,
                                   passes, which == VS_FILM_DISPLAY, s->exposed.ptr, nullptr, st),
                    "picture");
            src = s->exposed.ptr;
        }
        VS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "film copy");
    } else if (which == VS_FILM_RGBA8) {
        if (bytes != npix * 4) return fail(ctx, VS_E_INVALID, "film size mismatch");
        uchar4 *out8 = reinterpret_cast<uchar4 *>(s->exposed.ptr);
        VS_CUDA(launch_picture(s->film32.ptr, static_cast<uint32_t>(npix), s->host.cam.exposure, s->host.tone_mapper, 2u,
                               true, nullptr, out8, st),
                "picture");
        VS_CUDA(cudaMemcpyAsync(dst, out8, bytes, cudaMemcpyDeviceToHost, st), "film copy");
    } else if (which == VS_FILM_SUM64) {
        if (!s->film64_valid) return fail(ctx, VS_E_STATE, "FP64 film not rendered");
        if (bytes != npix * 32) return fail(ctx, VS_E_INVALID, "film size mismatch");
        VS_CUDA(cudaMemcpyAsync(dst, s->film64.ptr, bytes, cudaMemcpyDeviceToHost, st), "film copy");
    } else if (which == VS_FILM_SUMSQ64) {
        if (!s->film64sq_valid) return fail(ctx, VS_E_STATE, "FP64 film with squares not rendered (vs_render, FP64)");
        if (bytes != npix * 32) return fail(ctx, VS_E_INVALID, "film size mismatch");
        VS_CUDA(cudaMemcpyAsync(dst, s->film64.ptr + npix * 4, bytes, cudaMemcpyDeviceToHost, st), "film copy");
    } else {
        return fail(ctx, VS_E_INVALID, "unknown film buffer");
    }
    VS_CUDA(cudaStreamSynchronize(st), "film sync");
    return VS_OK;
}

int vs_trace_closest_device(vs_scene *s, const float *rays, uint32_t n, vs_hit *hits, float *t, void *stream) {
    if (!s || (n && (!rays || !hits || !t))) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot trace");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede tracing");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(launch_trace_closest(s->device_view(), rays, n, reinterpret_cast<Hit *>(hits), t, pick_stream(s, stream)),
            "trace launch");
    return VS_OK;
}

int vs_trace_any_device(vs_scene *s, const float *rays, uint32_t n, uint32_t *occ, void *stream) {
    if (!s || (n && (!rays || !occ))) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot trace");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede tracing");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(launch_trace_any(s->device_view(), rays, n, occ, pick_stream(s, stream)), "trace launch");
    return VS_OK;
}

int vs_trace_closest_host(vs_scene *s, const float *rays, uint32_t n, vs_hit *hits, float *t) {
    if (!s || (n && (!rays || !hits || !t))) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot trace");
    if (n == 0) return VS_OK;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    float *d_rays = nullptr, *d_t = nullptr;
    vs_hit *d_hits = nullptr;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMallocAsync(&d_rays, static_cast<size_t>(n) * 32, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_hits, static_cast<size_t>(n) * sizeof(vs_hit), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_t, static_cast<size_t>(n) * 4, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, static_cast<size_t>(n) * 32, cudaMemcpyHostToDevice, st);
    int rc = VS_OK;
    if (e == cudaSuccess) rc = vs_trace_closest_device(s, d_rays, n, d_hits, d_t, st);
    if (e == cudaSuccess && rc == VS_OK) e = cudaMemcpyAsync(hits, d_hits, static_cast<size_t>(n) * sizeof(vs_hit), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && rc == VS_OK) e = cudaMemcpyAsync(t, d_t, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, st);
    if (d_rays) cudaFreeAsync(d_rays, st);
    if (d_hits) cudaFreeAsync(d_hits, st);
    if (d_t) cudaFreeAsync(d_t, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace (host buffers)");
    if (rc != VS_OK) return rc;
    if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "trace sync");
    return VS_OK;
}

int vs_trace_any_host(vs_scene *s, const float *rays, uint32_t n, uint32_t *occ) {
    if (!s || (n && (!rays || !occ))) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot trace");
    if (n == 0) return VS_OK;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    float *d_rays = nullptr;
    uint32_t *d_occ = nullptr;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMallocAsync(&d_rays, static_cast<size_t>(n) * 32, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_occ, static_cast<size_t>(n) * 4, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, static_cast<size_t>(n) * 32, cudaMemcpyHostToDevice, st);
    int rc = VS_OK;
    if (e == cudaSuccess) rc = vs_trace_any_device(s, d_rays, n, d_occ, st);
    if (e == cudaSuccess && rc == VS_OK) e = cudaMemcpyAsync(occ, d_occ, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, st);
    if (d_rays) cudaFreeAsync(d_rays, st);
    if (d_occ) cudaFreeAsync(d_occ, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace (host buffers)");
    if (rc != VS_OK) return rc;
    if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "trace sync");
    return VS_OK;
}

int vs_sampler_stream(vs_context *ctx, int kind, uint32_t seed, const uint32_t *keys4, uint32_t count, uint32_t draws,
                      float *out) {
    if (!ctx || (count && draws && (!keys4 || !out))) return fail(ctx, VS_E_INVALID, "null argument");
    if (kind != kSamplerIndependent && kind != kSamplerPCG)
        return fail(ctx, VS_E_INVALID, "sampler kind must be 0 (independent) or 1 (pcg)");
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot run kernels");
    if (count == 0 || draws == 0) return VS_OK;
    const size_t out_bytes = static_cast<size_t>(count) * draws * 4;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    uint4 *d_keys = nullptr;
    float *d_out = nullptr;
    cudaError_t e = cudaMallocAsync(&d_keys, static_cast<size_t>(count) * 16, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_out, out_bytes, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_keys, keys4, static_cast<size_t>(count) * 16, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_sampler_stream(d_keys, count, draws, static_cast<uint32_t>(kind), seed, d_out, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, st);
    if (d_keys) cudaFreeAsync(d_keys, st);
    if (d_out) cudaFreeAsync(d_out, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sampler stream");
    if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "sampler stream sync");
    return VS_OK;
}

uint64_t vs_launch_count(void) { return launch_count(); }

int vs_timing_enable(vs_scene *s, int enable) {
    if (!s) return VS_E_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    for (cudaEvent_t e : s->ev_render) cudaEventDestroy(e);
    for (cudaEvent_t e : s->ev_film) cudaEventDestroy(e);
    s->ev_render.clear();
    s->ev_film.clear();
    s->timing = enable != 0;
    return VS_OK;
}

int vs_timing_read(vs_scene *s, double *render_ms, double *film_ms, uint32_t *render_launches) {
    if (!s || !render_ms || !film_ms || !render_launches) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(s->mu);
    double r = 0.0, f = 0.0;
    for (size_t i = 0; i + 1 < s->ev_render.size(); i += 2) {
        float ms = 0.0f;
        VS_CUDA(cudaEventSynchronize(s->ev_render[i + 1]), "timing sync");
        VS_CUDA(cudaEventElapsedTime(&ms, s->ev_render[i], s->ev_render[i + 1]), "timing read");
        r += ms;
    }
    for (size_t i = 0; i + 1 < s->ev_film.size(); i += 2) {
        float ms = 0.0f;
        VS_CUDA(cudaEventSynchronize(s->ev_film[i + 1]), "timing sync");
        VS_CUDA(cudaEventElapsedTime(&ms, s->ev_film[i], s->ev_film[i + 1]), "timing read");
        f += ms;
    }
    *render_ms = r;
    *film_ms = f;
    *render_launches = static_cast<uint32_t>(s->ev_render.size() / 2);
    return VS_OK;
}

int vs_render_stats(vs_scene *s, uint32_t frame_begin, uint32_t frame_count, uint64_t *out3) {
    if (!s || !out3) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot render");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede vs_render_stats");
    if (has_mix(s->host)) return fail(ctx, VS_E_UNSUPPORTED, "mix / add materials in the instrumented render");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint64_t npix = static_cast<uint64_t>(s->host.cam.width) * s->host.cam.height;
    if (npix * frame_count > kMaxPathsPerLaunch) return fail(ctx, VS_E_RANGE, "too many paths for one instrumented launch");
    VS_CUDA(s->radiance.alloc(static_cast<size_t>(npix * frame_count)), "radiance alloc");
    unsigned long long *d_stats = nullptr;
    VS_CUDA(cudaMalloc(&d_stats, 3 * sizeof(unsigned long long)), "stats alloc");
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemsetAsync(d_stats, 0, 3 * sizeof(unsigned long long), st);
    DeviceScene dv = s->device_view();
    dv.stats = d_stats;
    if (e == cudaSuccess) e = launch_render(dv, frame_begin, frame_count, s->radiance.ptr, st);
    unsigned long long h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_stats, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_stats);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "instrumented render");
    out3[0] = h[0];
    out3[1] = h[1];
    out3[2] = h[2];
    return VS_OK;
}

}  // extern "C"

namespace {

static_assert(sizeof(RtParams) == VS_RESTIR_PARAMS_BYTES, "RtParams layout changed");

// General 4x4 inverse in double (Sensor::device_w2c = inverse(c2w), sensor.cpp:194-201).
m4 inverse4(const m4 &a) {
    double m[16], inv[16];
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) m[4 * c + r] = a.m[c][r];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    m4 r{};
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 4; ++k) r.m[c][k] = static_cast<float>(inv[4 * c + k] / det);
    return r;
}

// The parameter block of the next ReSTIR frame.
RtParams rt_params(const vs_scene *s, uint32_t frame) {
    const HostScene &h = s->host;
    RtParams p{};
    p.di = h.rt_di;
    p.gi = h.rt_gi;
    p.M_light = h.rt_M_light;
    p.M_bsdf = h.rt_M_bsdf;
    p.max_recursion = h.rt_max_recursion;
    p.pairwise = h.rt_pairwise;
    p.gi_max_depth = h.ip.max_depth;
    p.frame = frame;
    p.width = h.cam.width;
    p.height = h.cam.height;
    p.w2c = inverse4(h.cam.c2w);
    p.view_pos = make3(h.cam.c2w.m[3][0], h.cam.c2w.m[3][1], h.cam.c2w.m[3][2]);
    bool prev = s->rt.have_prev && s->rt.width == h.cam.width && s->rt.height == h.cam.height;
    p.prev_cam = prev ? s->rt.prev_cam : h.cam;
    p.prev_w2c = prev ? s->rt.prev_w2c : p.w2c;
    p.prev_view_pos = prev ? s->rt.prev_pos : p.view_pos;
    p.di_factor = h.rt_di.open ? 1.0f : 0.0f;
    p.gi_factor = h.rt_gi.open ? 1.0f : 0.0f;
    return p;
}

int rt_ensure(vs_scene *s, cudaStream_t st) {
    vs_context *ctx = s->ctx;
    vs_scene::Rt &r = s->rt;
    uint32_t w = s->host.cam.width, hgt = s->host.cam.height;
    if (r.width == w && r.height == hgt && r.surf[0].ptr) return VS_OK;
    size_t n = static_cast<size_t>(w) * hgt;
    r.free();
    for (int k = 0; k < 2; ++k) {
        VS_CUDA(r.surf[k].alloc(n), "restir alloc");
        VS_CUDA(r.ext[k].alloc(n), "restir alloc");
        VS_CUDA(r.di[k].alloc(n), "restir alloc");
        VS_CUDA(r.gi[k].alloc(n), "restir alloc");
    }
    VS_CUDA(r.hit_bsdf.alloc(n), "restir alloc");
    VS_CUDA(r.motion.alloc(n), "restir alloc");
    VS_CUDA(r.di_pass.alloc(n), "restir alloc");
    VS_CUDA(r.gi_pass.alloc(n), "restir alloc");
    VS_CUDA(r.gi_init.alloc(n), "restir alloc");
    VS_CUDA(r.di_radiance.alloc(n), "restir alloc");
    VS_CUDA(r.gi_radiance.alloc(n), "restir alloc");
    VS_CUDA(r.di_stage.alloc(4 * n), "restir alloc");
    VS_CUDA(r.di_ray.alloc(2 * n), "restir alloc");
    VS_CUDA(r.di_hit.alloc(n), "restir alloc");
    VS_CUDA(r.di_list.alloc(n), "restir alloc");
    VS_CUDA(r.di_count.alloc(3), "restir alloc");
    VS_CUDA(r.gs_nb.alloc(n * kMaxSpatialNeighbours), "restir alloc");
    VS_CUDA(r.gs_ray.alloc(2 * n * kMaxSpatialNeighbours), "restir alloc");
    VS_CUDA(r.gs_vis.alloc(n * kMaxSpatialNeighbours), "restir alloc");
    VS_CUDA(r.gs_list.alloc(n * kMaxSpatialNeighbours), "restir alloc");
    VS_CUDA(r.gs_count.alloc(2), "restir alloc");
    r.width = w;
    r.height = hgt;
    r.have_prev = false;
    r.rendered = false;
    VS_CUDA(rt_all::launch_rt_reset(static_cast<uint32_t>(n), r.view(), st), "restir reset");
    add_launches(1);
    return VS_OK;
}

// Clears the denoiser's history: SVGFData and history lengths to zero, the
// G-buffer to PixelGeometry's defaults (linear depth -1: nothing to
// reproject from).
int svgf_reset(vs_scene *s, cudaStream_t st) {
    vs_context *ctx = s->ctx;
    vs_scene::Svgf &v = s->svgf;
    const size_t n = static_cast<size_t>(v.width) * v.height;
    if (n == 0) return VS_OK;
    std::vector<SvgfGeom> g(n, SvgfGeom{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f});
    for (int k = 0; k < 2; ++k) {
        VS_CUDA(cudaMemcpyAsync(v.geom[k].ptr, g.data(), n * sizeof(SvgfGeom), cudaMemcpyHostToDevice, st),
                "svgf reset");
        VS_CUDA(cudaMemsetAsync(v.history[k].ptr, 0, n * sizeof(float), st), "svgf reset");
    }
    for (int k = 0; k < 3; ++k) VS_CUDA(cudaMemsetAsync(v.data[k].ptr, 0, n * sizeof(SvgfData), st), "svgf reset");
    VS_CUDA(cudaStreamSynchronize(st), "svgf reset");
    v.prev = 0;
    v.rendered = false;
    return VS_OK;
}

int svgf_ensure(vs_scene *s, cudaStream_t st) {
    vs_context *ctx = s->ctx;
    vs_scene::Svgf &v = s->svgf;
    const uint32_t w = s->host.cam.width, h = s->host.cam.height;
    if (v.width == w && v.height == h && v.out.ptr) return VS_OK;
    const size_t n = static_cast<size_t>(w) * h;
    v.free();
    for (int k = 0; k < 2; ++k) {
        VS_CUDA(v.geom[k].alloc(n), "svgf alloc");
        VS_CUDA(v.history[k].alloc(n), "svgf alloc");
    }
    for (int k = 0; k < 3; ++k) VS_CUDA(v.data[k].alloc(n), "svgf alloc");
    VS_CUDA(v.motion.alloc(n), "svgf alloc");
    VS_CUDA(v.albedo.alloc(n), "svgf alloc");
    VS_CUDA(v.emission.alloc(n), "svgf alloc");
    VS_CUDA(v.out.alloc(n), "svgf alloc");
    v.width = w;
    v.height = h;
    return svgf_reset(s, st);
}

// One ReSTIR frame on `st`; the caller holds s->mu and has checked the
// scene.  `launches` gets the kernels launched.
int restir_frame_locked(vs_scene *s, uint32_t frame_index, uint32_t film_index, cudaStream_t st,
                        unsigned *launches) {
    vs_context *ctx = s->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    int rc = ensure_film(s);
    if (rc != VS_OK) return rc;
    rc = rt_ensure(s, st);
    if (rc != VS_OK) return rc;
    RtParams p = rt_params(s, frame_index);
    auto timed_event = [&](std::vector<cudaEvent_t> &v) -> cudaError_t {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        v.push_back(e);
        return cudaEventRecord(e, st);
    };
    if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
    unsigned n = 0;
    const uint64_t rt_npix = static_cast<uint64_t>(p.width) * p.height;
    const bool wavefront = s->schedule == VS_SCHEDULE_WAVEFRONT && rt_npix <= kWfWaveSlots;
    WfBuffers wfv{};
    if (wavefront) {
        VS_CUDA(s->wf.ensure(static_cast<uint32_t>(rt_npix), false), "wavefront slots alloc");
        VS_CUDA(s->radiance.alloc(rt_npix), "radiance alloc");
        wfv = s->wf.view();
    }
    // Scenes of diffuse surfaces and emitters only take the kernels compiled
    // for those materials alone.
    const uint32_t classes = shading_classes(s->host);
    const uint32_t diffuse_only = 1u | (1u << (1u + kMatDiffuse)) | (1u << (1u + kMatBlackBody));
    auto launch = (classes & ~diffuse_only) == 0u ? rt_diffuse::launch_rt_frame : rt_all::launch_rt_frame;
    VS_CUDA(launch(s->device_view(), p, s->rt.view(), film_index, s->film32.ptr, wavefront ? &wfv : nullptr,
                   wavefront ? s->radiance.ptr : nullptr, classes, st, &n),
            "restir launch");
    add_launches(n);
    if (launches) *launches += n;
    if (s->svgf.on) {
        // The denoiser over the frame's film (SVGF::dispatch after the combine, rt.cpp:157-158).
        rc = svgf_ensure(s, st);
        if (rc != VS_OK) return rc;
        unsigned m = 0;
        uint32_t final_d = 0;
        VS_CUDA(launch_svgf(s->device_view(), p, s->host.svgf, s->svgf.view(s->film32.ptr), s->svgf.prev, &final_d, st,
                            &m),
                "svgf launch");
        s->svgf.prev = final_d;
        s->svgf.rendered = true;
        add_launches(m);
        if (launches) *launches += m;
    }
    if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
    if (st != ctx->stream) {
        if (!s->ev_join) VS_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming), "join event");
        VS_CUDA(cudaEventRecord(s->ev_join, st), "join record");
        VS_CUDA(cudaStreamWaitEvent(ctx->stream, s->ev_join, 0), "join wait");
    }
    // Sensor::after_render -> store_prev_data (sensor.cpp:95-103).
    s->rt.prev_cam = s->host.cam;
    s->rt.prev_w2c = p.w2c;
    s->rt.prev_pos = p.view_pos;
    s->rt.have_prev = true;
    s->rt.last = p;
    s->rt.rendered = true;
    s->film_frames = film_index + 1u;
    s->film64_valid = false;
    s->film64sq_valid = false;
    return VS_OK;
}

// The per-pixel buffers a real-time frame uses, allocated up front so that a
// server can count them and its scheduler allocates nothing; the caller holds
// s->mu.
int restir_prepare_locked(vs_scene *s) {
    vs_context *ctx = s->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    int rc = ensure_film(s);
    if (rc != VS_OK) return rc;
    rc = rt_ensure(s, ctx->stream);
    if (rc != VS_OK) return rc;
    const uint64_t npix = static_cast<uint64_t>(s->host.cam.width) * s->host.cam.height;
    if (s->schedule == VS_SCHEDULE_WAVEFRONT && npix <= kWfWaveSlots) {
        VS_CUDA(s->wf.ensure(static_cast<uint32_t>(npix), false), "wavefront slots alloc");
        VS_CUDA(s->radiance.alloc(npix), "radiance alloc");
    }
    if (s->svgf.on) {
        rc = svgf_ensure(s, ctx->stream);
        if (rc != VS_OK) return rc;
    }
    VS_CUDA(cudaStreamSynchronize(ctx->stream), "restir prepare");
    return VS_OK;
}

}  // namespace

extern "C" {

int vs_restir_frame(vs_scene *s, uint32_t frame_index, uint32_t film_index, void *stream) {
    if (!s) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot render");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede vs_restir_frame");
    if (!s->host.rt) return fail(ctx, VS_E_STATE, "scene integrator is not \"rt\"");
    if (film_index != 0 && film_index != s->film_frames)
        return fail(ctx, VS_E_STATE, "film_index must continue the film or restart at 0");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    return restir_frame_locked(s, frame_index, film_index, pick_stream(s, stream), nullptr);
}

int vs_restir_reset(vs_scene *s) {
    if (!s) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(s->mu);
    s->rt.have_prev = false;
    s->rt.rendered = false;
    if (ctx->device < 0 || !s->rt.surf[0].ptr) return VS_OK;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    size_t n = static_cast<size_t>(s->rt.width) * s->rt.height;
    VS_CUDA(rt_all::launch_rt_reset(static_cast<uint32_t>(n), s->rt.view(), ctx->stream), "restir reset");
    add_launches(1);
    return svgf_reset(s, ctx->stream);
}

int vs_restir_params(const vs_scene *s, uint32_t frame_index, void *dst, size_t bytes) {
    if (!s || !dst) return VS_E_INVALID;
    if (bytes != sizeof(RtParams)) return fail(s->ctx, VS_E_INVALID, "params size mismatch");
    if (!s->host.rt) return fail(s->ctx, VS_E_STATE, "scene integrator is not \"rt\"");
    RtParams p = rt_params(s, frame_index);
    std::memcpy(dst, &p, sizeof(p));
    return VS_OK;
}

int vs_restir_download(vs_scene *s, int which, void *dst, size_t bytes) {
    if (!s || !dst) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context has no ReSTIR buffers");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->rt.rendered) return fail(ctx, VS_E_STATE, "no ReSTIR frame rendered");
    size_t n = static_cast<size_t>(s->rt.width) * s->rt.height;
    uint32_t cur = (s->rt.last.frame + 1u) & 1u;
    const void *src = nullptr;
    size_t elem = 0;
    switch (which) {
        case VS_RESTIR_DI_RADIANCE: src = s->rt.di_radiance.ptr; elem = 16; break;
        case VS_RESTIR_GI_RADIANCE: src = s->rt.gi_radiance.ptr; elem = 16; break;
        case VS_RESTIR_MOTION: src = s->rt.motion.ptr; elem = 8; break;
        case VS_RESTIR_SURFACES: src = s->rt.surf[cur].ptr; elem = sizeof(RtSurface); break;
        case VS_RESTIR_DI_RESERVOIRS: src = s->rt.di[cur].ptr; elem = sizeof(DiReservoir); break;
        case VS_RESTIR_GI_RESERVOIRS: src = s->rt.gi[cur].ptr; elem = sizeof(GiReservoir); break;
        case VS_RESTIR_HIT_BSDF: src = s->rt.hit_bsdf.ptr; elem = sizeof(RtHitBsdf); break;
        case VS_RESTIR_GI_SAMPLES: src = s->rt.gi_init.ptr; elem = sizeof(GiReservoir); break;
        case VS_RESTIR_DENOISED:
        case VS_RESTIR_GBUFFER:
        case VS_RESTIR_SVGF_ALBEDO:
        case VS_RESTIR_SVGF_EMISSION:
        case VS_RESTIR_SVGF_DATA:
        case VS_RESTIR_SVGF_MOTION:
        case VS_RESTIR_SVGF_HISTORY: {
            if (!s->svgf.rendered) return fail(ctx, VS_E_STATE, "no frame rendered with the denoiser");
            const vs_scene::Svgf &v = s->svgf;
            if (which == VS_RESTIR_DENOISED) { src = v.out.ptr; elem = 16; }
            if (which == VS_RESTIR_GBUFFER) { src = v.geom[cur].ptr; elem = sizeof(SvgfGeom); }
            if (which == VS_RESTIR_SVGF_ALBEDO) { src = v.albedo.ptr; elem = 16; }
            if (which == VS_RESTIR_SVGF_EMISSION) { src = v.emission.ptr; elem = 16; }
            if (which == VS_RESTIR_SVGF_DATA) { src = v.data[v.prev].ptr; elem = sizeof(SvgfData); }
            if (which == VS_RESTIR_SVGF_MOTION) { src = v.motion.ptr; elem = 8; }
            if (which == VS_RESTIR_SVGF_HISTORY) { src = v.history[cur].ptr; elem = 4; }
            break;
        }
        default: return fail(ctx, VS_E_INVALID, "unknown ReSTIR buffer");
    }
    if (bytes != n * elem) return fail(ctx, VS_E_INVALID, "ReSTIR buffer size mismatch");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), "restir copy");
    VS_CUDA(cudaStreamSynchronize(ctx->stream), "restir sync");
    return VS_OK;
}

int vs_denoiser_enable(vs_scene *s, int on) {
    if (!s) return VS_E_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->host.rt) return fail(s->ctx, VS_E_STATE, "scene integrator is not \"rt\"");
    s->svgf.on = on != 0;
    return VS_OK;
}

int vs_denoiser_params(const vs_scene *s, void *dst, size_t bytes) {
    if (!s || !dst) return VS_E_INVALID;
    if (bytes != sizeof(SvgfParams)) return fail(s->ctx, VS_E_INVALID, "denoiser params size mismatch");
    std::lock_guard<std::mutex> lock(const_cast<vs_scene *>(s)->mu);
    if (!s->host.rt) return fail(s->ctx, VS_E_STATE, "scene integrator is not \"rt\"");
    std::memcpy(dst, &s->host.svgf, sizeof(SvgfParams));
    return VS_OK;
}

}  // extern "C"

struct vs_server {
    vs_context *ctx = nullptr;
    Server *impl = nullptr;
    std::mutex mu;
    std::string error;
    int fail(int code, const std::string &msg) {
        std::lock_guard<std::mutex> lk(mu);
        error = msg;
        return code;
    }
};

extern "C" {

int vs_server_create(vs_context *ctx, uint64_t hbm_budget, uint32_t max_jobs, uint64_t paths_per_batch,
                     vs_server **out) {
    if (!ctx || !out) return VS_E_INVALID;
    *out = nullptr;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot serve");
    std::string err;
    Server *impl = nullptr;
    int rc = server_create(ctx->device, hbm_budget, max_jobs, paths_per_batch, &impl, err);
    if (rc != VS_OK) return fail(ctx, rc, err);
    vs_server *s = new vs_server();
    s->ctx = ctx;
    s->impl = impl;
    *out = s;
    return VS_OK;
}

void vs_server_destroy(vs_server *s) {
    if (!s) return;
    server_destroy(s->impl);
    delete s;
}

int vs_server_add_scene(vs_server *s, vs_scene *scene, uint32_t *scene_id) {
    if (!s || !scene || !scene_id) return VS_E_INVALID;
    DeviceScene dv;
    uint64_t bytes = 0;
    bool rt = false;
    Camera cam{};
    const float4 *film = nullptr;
    {
        std::lock_guard<std::mutex> lock(scene->mu);
        if (!scene->uploaded) return s->fail(VS_E_STATE, "vs_scene_build_accel must precede vs_server_add_scene");
        if (scene->ctx->device != s->ctx->device) return s->fail(VS_E_INVALID, "scene on another device");
        rt = scene->host.rt;
        if (rt) {
            // The real-time buffers are allocated now and stay resident: the
            // scheduler allocates nothing and the budget counts them.
            int rc = restir_prepare_locked(scene);
            if (rc != VS_OK) return s->fail(rc, vs_last_error(scene->ctx));
            bytes = scene->device_bytes() + scene->rt_resident_bytes();
            cam = scene->host.cam;
            film = scene->film32.ptr;
        } else {
            dv = scene->device_view();
            bytes = scene->device_bytes();
        }
    }
    std::string err;
    int rc;
    if (rt) {
        RtServeHooks hooks;
        hooks.film = film;
        // One frame with the job's sensor, under the scene's lock.  The
        // scene's camera becomes the job's, so the frame's motion vectors and
        // temporal reuse see the previous frame's camera (the last job's).
        hooks.frame = [scene](const Camera &c, uint32_t frame, uint32_t film_index, cudaStream_t st,
                              unsigned *launches, std::string &e) {
            std::lock_guard<std::mutex> lock(scene->mu);
            scene->host.cam = c;
            int r = restir_frame_locked(scene, frame, film_index, st, launches);
            if (r != VS_OK) e = vs_last_error(scene->ctx);
            return r;
        };
        rc = server_add_rt_scene(s->impl, cam, bytes, std::move(hooks), scene_id, err);
    } else {
        rc = server_add_scene(s->impl, dv, bytes, scene_id, err);
    }
    return rc == VS_OK ? VS_OK : s->fail(rc, err);
}

int vs_server_submit(vs_server *s, const vs_job_desc *job, uint64_t *job_id) {
    if (!s || !job || !job_id) return VS_E_INVALID;
    if (job->width == 0 || job->height == 0 || job->spp == 0) return s->fail(VS_E_INVALID, "empty job");
    ServeJob j{};
    j.scene = job->scene;
    j.frame_begin = job->frame_begin;
    j.spp = job->spp;
    std::string err;
    // The job's sensor: the scene's camera at the job's resolution, with the
    // job's transform and field of view when given.
    const Camera *base = nullptr;
    int rc = server_scene_camera(s->impl, job->scene, &base, err);
    if (rc != VS_OK) return s->fail(rc, err);
    Camera cam = camera_at_resolution(*base, job->width, job->height);
    if (job->use_c2w)
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) cam.c2w.m[c][r] = job->c2w[4 * c + r];
    if (job->fov_y_deg > 0.0f) {
        float fov = std::min(std::max(job->fov_y_deg, 15.0f), 120.0f);
        cam.tan_half_fov = std::tan(fov * kPi / 180.0f * 0.5f);
    }
    j.cam = cam;
    rc = server_submit(s->impl, j, job_id, err);
    return rc == VS_OK ? VS_OK : s->fail(rc, err);
}

int vs_server_poll(vs_server *s, uint64_t job_id, int *done) {
    if (!s || !done) return VS_E_INVALID;
    std::string err;
    int rc = server_poll(s->impl, job_id, done, err);
    return rc == VS_OK ? VS_OK : s->fail(rc, err);
}

int vs_server_result(vs_server *s, uint64_t job_id, float *dst, size_t bytes, double timeout_s) {
    if (!s || !dst) return VS_E_INVALID;
    std::string err;
    int rc = server_result(s->impl, job_id, dst, bytes, timeout_s, err);
    return rc == VS_OK ? VS_OK : s->fail(rc, err);
}

int vs_server_stats_get(vs_server *s, vs_server_stats *out) {
    if (!s || !out) return VS_E_INVALID;
    ServeStats st;
    server_stats(s->impl, &st);
    out->submitted = st.submitted;
    out->completed = st.completed;
    out->batches = st.batches;
    out->graph_launches = st.graph_launches;
    out->kernel_launches = st.kernel_launches;
    out->paths = st.paths;
    out->wall_s = st.wall_s;
    out->gpu_busy_s = st.gpu_busy_s;
    out->p50_ms = st.p50_ms;
    out->p95_ms = st.p95_ms;
    out->p99_ms = st.p99_ms;
    out->mean_ms = st.mean_ms;
    out->max_ms = st.max_ms;
    out->peak_bytes = st.peak_bytes;
    out->peak_jobs = st.peak_jobs;
    out->resident_bytes = st.resident_bytes;
    out->scratch_bytes = st.scratch_bytes;
    return VS_OK;
}

const char *vs_server_last_error(const vs_server *s) {
    if (!s) return "null server";
    return s->error.c_str();
}

}  // extern "C"

struct vs_cache {
    vs_context *ctx = nullptr;
    MlpState st{};
    MlpAdam adam{1e-3f, 0.9f, 0.999f, 1e-8f, 1u, 0.0f};
    ~vs_cache() {
        if (ctx && ctx->device >= 0) cudaSetDevice(ctx->device);
        cudaFree(st.w);
        cudaFree(st.pack);
        cudaFree(st.m);
        cudaFree(st.v);
        cudaFree(st.grad);
        cudaFree(st.loss);
        cudaFree(st.err);
    }
};

namespace {
int cache_check_err(vs_cache *c) {
    vs_context *ctx = c->ctx;
    int h = 0;
    VS_CUDA(cudaMemcpy(&h, c->st.err, sizeof(int), cudaMemcpyDeviceToHost), "cache error flag");
    if (h) return fail(ctx, VS_E_CUDA, "tensor-core wait timed out in the radiance-cache kernels");
    return VS_OK;
}
}  // namespace

extern "C" {

int vs_cache_create(vs_context *ctx, uint64_t seed, vs_cache **out) {
    if (!ctx || !out) return VS_E_INVALID;
    *out = nullptr;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context has no radiance cache");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    vs_cache *c = new vs_cache();
    c->ctx = ctx;
    MlpState &s = c->st;
    cudaError_t e = cudaMalloc(&s.w, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMalloc(&s.pack, sizeof(uint16_t) * kMlpPackElems);
    if (e == cudaSuccess) e = cudaMalloc(&s.m, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMalloc(&s.v, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMalloc(&s.grad, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMalloc(&s.loss, sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s.err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s.pack, 0, sizeof(uint16_t) * kMlpPackElems);
    if (e == cudaSuccess) e = cudaMemset(s.m, 0, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(s.v, 0, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(s.grad, 0, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(s.loss, 0, sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(s.err, 0, sizeof(int));
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(ctx, e, "cache alloc");
    }
    // Uniform +-sqrt(6 / fan_in) from a splitmix64 stream.
    std::vector<float> w(kMlpParams);
    uint64_t x = seed;
    for (int i = 0; i < kMlpParams; ++i) {
        x += 0x9e3779b97f4a7c15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        float u = static_cast<float>(z >> 40) * (1.0f / 16777216.0f);
        w[i] = (2.0f * u - 1.0f) * std::sqrt(6.0f / 64.0f);
    }
    e = cudaMemcpy(s.w, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = mlp_pack(s, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(ctx, e, "cache init");
    }
    add_launches(1);
    *out = c;
    return VS_OK;
}

void vs_cache_destroy(vs_cache *c) { delete c; }

int vs_cache_get_weights(vs_cache *c, float *w, size_t count) {
    if (!c || !w || count != static_cast<size_t>(kMlpParams)) return VS_E_INVALID;
    vs_context *ctx = c->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(cudaDeviceSynchronize(), "cache sync");
    VS_CUDA(cudaMemcpy(w, c->st.w, sizeof(float) * count, cudaMemcpyDeviceToHost), "cache weights");
    return VS_OK;
}

int vs_cache_set_weights(vs_cache *c, const float *w, size_t count) {
    if (!c || !w || count != static_cast<size_t>(kMlpParams)) return VS_E_INVALID;
    vs_context *ctx = c->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(cudaDeviceSynchronize(), "cache sync");
    VS_CUDA(cudaMemcpy(c->st.w, w, sizeof(float) * count, cudaMemcpyHostToDevice), "cache weights");
    VS_CUDA(cudaMemset(c->st.m, 0, sizeof(float) * count), "cache moments");
    VS_CUDA(cudaMemset(c->st.v, 0, sizeof(float) * count), "cache moments");
    VS_CUDA(mlp_pack(c->st, nullptr), "cache pack");
    VS_CUDA(cudaDeviceSynchronize(), "cache sync");
    add_launches(1);
    c->adam.step = 1;
    return VS_OK;
}

int vs_cache_set_optimizer(vs_cache *c, float lr, float beta1, float beta2, float eps) {
    if (!c) return VS_E_INVALID;
    c->adam.lr = lr;
    c->adam.beta1 = beta1;
    c->adam.beta2 = beta2;
    c->adam.eps = eps;
    return VS_OK;
}

int vs_cache_infer(vs_cache *c, const uint16_t *features, uint32_t n, float *out4, void *stream) {
    if (!c || (n && (!features || !out4))) return VS_E_INVALID;
    vs_context *ctx = c->ctx;
    if ((reinterpret_cast<uintptr_t>(features) & 15u) || (reinterpret_cast<uintptr_t>(out4) & 15u))
        return fail(ctx, VS_E_INVALID, "cache buffers must be 16-byte aligned");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    VS_CUDA(mlp_infer(c->st, features, n, reinterpret_cast<float4 *>(out4), st), "cache infer");
    if (n) add_launches(1);
    return VS_OK;
}

int vs_cache_train(vs_cache *c, const uint16_t *features, const float *targets4, uint32_t n, int update,
                   void *stream) {
    if (!c || (n && (!features || !targets4))) return VS_E_INVALID;
    vs_context *ctx = c->ctx;
    if ((reinterpret_cast<uintptr_t>(features) & 15u) || (reinterpret_cast<uintptr_t>(targets4) & 15u))
        return fail(ctx, VS_E_INVALID, "cache buffers must be 16-byte aligned");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    c->adam.loss_scale = n ? 1.0f / (3.0f * static_cast<float>(n)) : 0.0f;
    VS_CUDA(mlp_train_step(c->st, features, reinterpret_cast<const float4 *>(targets4), n, c->adam, update != 0, st),
            "cache train");
    add_launches((n ? 1u : 0u) + (update ? 1u : 0u));
    if (update) c->adam.step += 1;
    return VS_OK;
}

int vs_cache_gradient(vs_cache *c, float *grad, size_t count, double *loss) {
    if (!c || !grad || !loss || count != static_cast<size_t>(kMlpParams)) return VS_E_INVALID;
    vs_context *ctx = c->ctx;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(cudaDeviceSynchronize(), "cache sync");
    int rc = cache_check_err(c);
    if (rc != VS_OK) return rc;
    VS_CUDA(cudaMemcpy(grad, c->st.grad, sizeof(float) * count, cudaMemcpyDeviceToHost), "cache gradient");
    VS_CUDA(cudaMemcpy(loss, c->st.loss, sizeof(double), cudaMemcpyDeviceToHost), "cache loss");
    return VS_OK;
}

int vs_render_cached(vs_scene *s, vs_cache *c, uint32_t frame_begin, uint32_t frame_count, uint32_t train_samples,
                     int film_precision, void *stream) {
    if (!s || !c) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot render");
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->uploaded) return fail(ctx, VS_E_STATE, "vs_scene_build_accel must precede vs_render_cached");
    const HostScene &h = s->host;
    if (h.ip.spectrum_dim != 3)
        return fail(ctx, VS_E_UNSUPPORTED, "cache rendering needs 3 hero wavelengths (the cache's 3 outputs)");
    if (has_mix(h)) return fail(ctx, VS_E_UNSUPPORTED, "mix / add materials in cache rendering");
    if (frame_begin != 0 && frame_begin != s->film_frames)
        return fail(ctx, VS_E_STATE, "frames must continue the film (frame_begin == frames rendered) or restart at 0");
    if (film_precision == VS_FILM_FP64 && frame_begin != 0 && !s->film64_valid)
        return fail(ctx, VS_E_STATE, "FP64 film must be enabled from frame 0");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = pick_stream(s, stream);
    int rc = ensure_film(s);
    if (rc != VS_OK) return rc;
    const uint32_t npix = h.cam.width * h.cam.height;
    if (train_samples > npix) train_samples = npix;
    if (film_precision == VS_FILM_FP64) VS_CUDA(s->film64.alloc(static_cast<size_t>(npix) * 8), "film64 alloc");
    vs_scene::CacheBufs &b = s->cachebuf;
    const size_t nt = train_samples ? train_samples : 1;
    VS_CUDA(b.q_feat.alloc(static_cast<size_t>(npix) * 64), "cache alloc");
    VS_CUDA(b.q_rec.alloc(npix), "cache alloc");
    VS_CUDA(b.q_out.alloc(npix), "cache alloc");
    VS_CUDA(b.t_feat.alloc(nt * 64), "cache alloc");
    VS_CUDA(b.b_feat.alloc(nt * 64), "cache alloc");
    VS_CUDA(b.t_rec.alloc(nt), "cache alloc");
    VS_CUDA(b.b_out.alloc(nt), "cache alloc");
    VS_CUDA(b.targets.alloc(nt), "cache alloc");
    if (!b.mat.ptr) {
        // Albedo (the colour slot's RGB) and roughness (alpha; 1 for diffuse
        // and emitters) of every material, for the feature encoding.
        std::vector<float4> m(h.materials.size());
        for (size_t i = 0; i < m.size(); ++i) {
            const Material &mt = h.materials[i];
            f3 rgb = i < h.material_rgb.size() ? h.material_rgb[i] : make3(0.0f);
            float rough = (mt.type == kMatDiffuse || mt.type == kMatBlackBody) ? 1.0f : mt.p[0];
            m[i] = make_float4(rgb.x, rgb.y, rgb.z, rough);
        }
        VS_CUDA(b.mat.upload(m), "cache materials");
    }
    f3 lo = make3(3.0e38f), hi = make3(-3.0e38f);
    for (const f3 &q : h.pos) {
        lo = vmin(lo, q);
        hi = vmax(hi, q);
    }
    CacheFrameParams p{};
    p.bmin = lo;
    f3 ext = hi - lo;
    p.binv = make3(ext.x > 0 ? 1.0f / ext.x : 0.0f, ext.y > 0 ? 1.0f / ext.y : 0.0f, ext.z > 0 ? 1.0f / ext.z : 0.0f);
    p.mat = b.mat.ptr;
    p.q_feat = b.q_feat.ptr;
    p.q_rec = b.q_rec.ptr;
    p.q_out = b.q_out.ptr;
    p.n_train = train_samples;
    p.train_stride = train_samples ? std::max<uint32_t>(1u, npix / train_samples) : 1u;
    p.t_feat = b.t_feat.ptr;
    p.b_feat = b.b_feat.ptr;
    p.t_rec = b.t_rec.ptr;
    p.b_out = b.b_out.ptr;
    p.targets = b.targets.ptr;
    p.query_depth = 2;
    p.suffix_depth = 2;
    // Wavefront frames need one path slot per pixel.
    const bool wavefront = s->schedule == VS_SCHEDULE_WAVEFRONT && npix <= kWfWaveSlots;
    if (wavefront) {
        VS_CUDA(s->wf.ensure(npix, false), "wavefront slots alloc");
        VS_CUDA(s->radiance.alloc(npix), "radiance alloc");
        VS_CUDA(b.suffix_list.alloc(nt), "cache alloc");
        VS_CUDA(b.suffix_count.alloc(1), "cache alloc");
    }
    DeviceScene dv = s->device_view();
    auto timed_event = [&](std::vector<cudaEvent_t> &v) -> cudaError_t {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        v.push_back(e);
        return cudaEventRecord(e, st);
    };
    for (uint32_t f = 0; f < frame_count; ++f) {
        const uint32_t frame = frame_begin + f;
        p.frame = frame;
        // Training pixels move every frame: offset from a hash of the frame index.
        uint32_t hsh = frame * 0x9e3779b9u;
        hsh ^= hsh >> 16;
        hsh *= 0x85ebca6bu;
        hsh ^= hsh >> 13;
        p.train_offset = train_samples ? hsh % p.train_stride : 0u;
        if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
        unsigned n = 0;
        double *f64 = film_precision == VS_FILM_FP64 ? s->film64.ptr : nullptr;
        if (wavefront) {
            VS_CUDA(launch_cache_frame_wavefront(dv, p, c->st, s->film32.ptr, f64, frame, s->wf.view(),
                                                 shading_classes(h), s->radiance.ptr, b.suffix_list.ptr,
                                                 b.suffix_count.ptr, st, &n),
                    "cache frame");
        } else {
            VS_CUDA(launch_cache_frame(dv, p, c->st, s->film32.ptr, f64, frame, st, &n), "cache frame");
        }
        add_launches(n);
        if (train_samples) {
            c->adam.loss_scale = 1.0f / (3.0f * static_cast<float>(train_samples));
            VS_CUDA(mlp_train_step(c->st, p.t_feat, p.targets, train_samples, c->adam, true, st), "cache train");
            c->adam.step += 1;
            add_launches(2);
        }
        if (s->timing) VS_CUDA(timed_event(s->ev_render), "timing event");
    }
    if (st != ctx->stream) {
        if (!s->ev_join) VS_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming), "join event");
        VS_CUDA(cudaEventRecord(s->ev_join, st), "join record");
        VS_CUDA(cudaStreamWaitEvent(ctx->stream, s->ev_join, 0), "join wait");
    }
    s->film_frames = frame_begin + frame_count;
    s->film64_valid = film_precision == VS_FILM_FP64 && (frame_begin == 0 || s->film64_valid);
    s->film64sq_valid = false;
    if (frame_count) {
        b.npix = npix;
        b.n_train = train_samples;
    }
    return VS_OK;
}

int vs_cache_download(vs_scene *s, int which, void *dst, size_t bytes) {
    if (!s || !dst) return VS_E_INVALID;
    vs_context *ctx = s->ctx;
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context has no cache buffers");
    std::lock_guard<std::mutex> lock(s->mu);
    const vs_scene::CacheBufs &b = s->cachebuf;
    if (b.npix == 0) return fail(ctx, VS_E_STATE, "no cache-terminated frame rendered");
    const void *src = nullptr;
    size_t n = 0, elem = 0;
    switch (which) {
        case VS_CACHE_QUERY_FEATURES: src = b.q_feat.ptr; n = b.npix; elem = 128; break;
        case VS_CACHE_QUERY_RECORDS: src = b.q_rec.ptr; n = b.npix; elem = sizeof(CacheQueryRec); break;
        case VS_CACHE_QUERY_OUTPUT: src = b.q_out.ptr; n = b.npix; elem = 16; break;
        case VS_CACHE_TRAIN_FEATURES: src = b.t_feat.ptr; n = b.n_train; elem = 128; break;
        case VS_CACHE_TRAIN_RECORDS: src = b.t_rec.ptr; n = b.n_train; elem = sizeof(CacheTrainRec); break;
        case VS_CACHE_SUFFIX_FEATURES: src = b.b_feat.ptr; n = b.n_train; elem = 128; break;
        case VS_CACHE_SUFFIX_OUTPUT: src = b.b_out.ptr; n = b.n_train; elem = 16; break;
        case VS_CACHE_TARGETS: src = b.targets.ptr; n = b.n_train; elem = 16; break;
        default: return fail(ctx, VS_E_INVALID, "unknown cache buffer");
    }
    if (bytes != n * elem) return fail(ctx, VS_E_INVALID, "cache buffer size mismatch");
    if (n == 0) return VS_OK;
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    VS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), "cache copy");
    VS_CUDA(cudaStreamSynchronize(ctx->stream), "cache sync");
    return VS_OK;
}

int vs_albedo_luts(int which, const char *cache_path, float *out, size_t count) {
    if (!out || count != static_cast<size_t>(kLutFloats)) return VS_E_INVALID;
    const float *t = which == 0 ? microfacet_luts() : regenerate_microfacet_luts(cache_path ? cache_path : "");
    std::memcpy(out, t, count * sizeof(float));
    return VS_OK;
}

int vs_albedo_luts_gpu(vs_context *ctx, uint32_t strata, float *out, size_t count) {
    if (!ctx) return VS_E_INVALID;
    if (!out || count != static_cast<size_t>(kLutFloats)) return fail(ctx, VS_E_INVALID, "out must hold the table floats");
    if (strata < 1u || strata > 4096u) return fail(ctx, VS_E_RANGE, "strata must be in [1, 4096]");
    if (ctx->device < 0) return fail(ctx, VS_E_NO_DEVICE, "host-only context cannot generate on the GPU");
    VS_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    struct Owned {
        DevBuf<float> b;
        ~Owned() { b.free(); }
    } d;
    VS_CUDA(d.b.alloc(count), "lut alloc");
    VS_CUDA(launch_albedo_luts(d.b.ptr, strata, ctx->stream), "albedo luts");
    VS_CUDA(cudaMemcpyAsync(out, d.b.ptr, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream), "lut copy");
    VS_CUDA(cudaStreamSynchronize(ctx->stream), "lut sync");
    return VS_OK;
}

int vs_rgb_to_spectrum(vs_context *ctx, const char *table_cache, const float *rgb3, int mode, float *out4) {
    if (!rgb3 || !out4) return fail(ctx, VS_E_INVALID, "null argument");
    const float *table = rgb2spec_table(table_cache ? table_cache : "");
    if (mode == 0) rgb2spec_decode_albedo(table, rgb3, out4);
    else if (mode == 1) rgb2spec_decode_unbound(table, rgb3, out4);
    else return fail(ctx, VS_E_INVALID, "mode must be 0 or 1");
    return VS_OK;
}

}  // extern "C"
