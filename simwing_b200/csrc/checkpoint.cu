// Structure::checkpoint / restore (src/fsi/structure.cpp:961-1027) for the
// device state: an opaque, checksummed little-endian byte image bound to the
// definition fingerprint.  Restoring an image taken from the same structure
// reproduces its state bit for bit (positions are stored as the frame
// origin plus the FP32 offsets, both exactly).
#include "structure_impl.h"

#include <cmath>
#include <cstring>

namespace swb {
namespace {

constexpr char kMagic[8] = {'S', 'W', 'B', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kVersion = 1;

struct Writer {
    std::vector<uint8_t> bytes;
    void raw(const void* p, size_t n) {
        const auto* c = static_cast<const uint8_t*>(p);
        bytes.insert(bytes.end(), c, c + n);
    }
    void u32(uint32_t v) { raw(&v, 4); }
    void u64(uint64_t v) { raw(&v, 8); }
    void f64(double v) { raw(&v, 8); }
};

struct Reader {
    const uint8_t* p;
    size_t n, at = 0;
    void raw(void* out, size_t k) {
        if (at + k > n) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: truncated");
        std::memcpy(out, p + at, k);
        at += k;
    }
    uint32_t u32() { uint32_t v; raw(&v, 4); return v; }
    uint64_t u64() { uint64_t v; raw(&v, 8); return v; }
    double f64() { double v; raw(&v, 8); return v; }
};

uint64_t fnv1a(const uint8_t* p, size_t n) {
    uint64_t h = 14695981039346656037ULL;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

std::vector<uint8_t> serialize(const StructureImpl& m) {
    std::vector<float4> pos, prev, vel;
    DevPayloadState pay{};
    double o[3];
    m.fetch(pos, prev, vel, pay, o);
    Writer w;
    w.raw(kMagic, 8);
    w.u32(kVersion);
    w.u32(m.def.has_suspension ? 1u : 0u);
    w.u64(m.fingerprint);
    w.u64(m.accepted);
    w.f64(m.time);
    w.f64(m.last_dt);
    w.f64(o[0]); w.f64(o[1]); w.f64(o[2]);
    const uint64_t N = m.def.nodes.size();
    w.u64(N);
    for (uint64_t n = 0; n < N; ++n) {
        const uint32_t s = m.slot_of_node[n];
        for (const float4* a : {&pos[s], &prev[s], &vel[s]}) {
            w.f64(a->x); w.f64(a->y); w.f64(a->z);
        }
    }
    for (const auto& f : m.pending) { w.f64(f.x); w.f64(f.y); w.f64(f.z); }
    w.f64(m.last_applied.x); w.f64(m.last_applied.y); w.f64(m.last_applied.z);
    w.u64(m.pressure.size());
    for (double p : m.pressure) w.f64(p);
    if (m.def.has_suspension) w.raw(&pay, sizeof(pay));
    const uint64_t sum = fnv1a(w.bytes.data(), w.bytes.size());
    w.u64(sum);
    return w.bytes;
}

bool is_finite_value(double v) { return std::isfinite(v); }

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

swb_status swb_structure_checkpoint_size(const swb_structure* s, uint64_t* bytes) {
    return guarded([&] {
        if (!s || !bytes) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        const uint64_t N = m.def.nodes.size();
        *bytes = 8 + 4 + 4 + 8 + 8 + 8 + 8 + 24 + 8 + N * 72 + N * 24 + 24 + 8 + m.pressure.size() * 8 +
                 (m.def.has_suspension ? sizeof(DevPayloadState) : 0) + 8;
    });
}

swb_status swb_structure_checkpoint(const swb_structure* s, void* buffer, uint64_t bytes) {
    return guarded([&] {
        if (!s || !buffer) raise(SWB_INVALID_ARGUMENT, "null argument");
        const std::vector<uint8_t> image = serialize(s->s);
        if (bytes != image.size()) raise(SWB_INVALID_ARGUMENT, "checkpoint buffer size mismatch");
        std::memcpy(buffer, image.data(), image.size());
    });
}

swb_status swb_structure_restore(swb_structure* s, const void* buffer, uint64_t bytes) {
    return guarded([&] {
        if (!s || !buffer) raise(SWB_INVALID_ARGUMENT, "null argument");
        StructureImpl& m = s->s;
        const auto* p = static_cast<const uint8_t*>(buffer);
        if (bytes < 16) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        uint64_t stored;
        std::memcpy(&stored, p + bytes - 8, 8);
        if (stored != fnv1a(p, bytes - 8)) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: checksum");
        Reader r{p, static_cast<size_t>(bytes - 8)};
        char magic[8];
        r.raw(magic, 8);
        if (std::memcmp(magic, kMagic, 8) != 0) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: magic");
        if (r.u32() != kVersion) raise(SWB_INVALID_ARGUMENT, "Unsupported structure checkpoint version");
        const bool susp = r.u32() != 0;
        if (r.u64() != m.fingerprint)
            raise(SWB_INVALID_ARGUMENT, "Structure checkpoint belongs to a different definition");
        if (susp != m.def.has_suspension) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        const uint64_t accepted = r.u64();
        const double time = r.f64();
        const double last_dt = r.f64();
        double o[3] = {r.f64(), r.f64(), r.f64()};
        const uint64_t N = r.u64();
        if (N != m.def.nodes.size() || !is_finite_value(time) || time < 0.0 || !is_finite_value(o[0]) || !is_finite_value(o[1]) || !is_finite_value(o[2]))
            raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        std::vector<float4> pos(N), prev(N), vel(N);
        for (uint64_t n = 0; n < N; ++n) {
            const uint32_t sl = m.slot_of_node[n];
            double v[9];
            for (double& x : v) {
                x = r.f64();
                if (!is_finite_value(x)) raise(SWB_INVALID_ARGUMENT, "Structure checkpoint is non-finite");
            }
            const float w = m.inv_mass[sl];
            pos[sl] = make_float4(v[0], v[1], v[2], w);
            prev[sl] = make_float4(v[3], v[4], v[5], w);
            vel[sl] = make_float4(v[6], v[7], v[8], 0.0f);
        }
        std::vector<swb_vec3> pending(N);
        for (auto& f : pending) {
            f.x = r.f64(); f.y = r.f64(); f.z = r.f64();
            if (!is_finite_value(f.x) || !is_finite_value(f.y) || !is_finite_value(f.z)) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        }
        swb_vec3 last{r.f64(), r.f64(), r.f64()};
        if (!is_finite_value(last.x) || !is_finite_value(last.y) || !is_finite_value(last.z)) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        const uint64_t T = r.u64();
        if (T != m.pressure.size()) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        std::vector<double> pressure(T);
        for (double& x : pressure) {
            x = r.f64();
            if (!is_finite_value(x)) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        }
        DevPayloadState pay{};
        if (susp) r.raw(&pay, sizeof(pay));
        if (r.at != r.n) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: trailing bytes");
        // commit
        cuda_check(cudaSetDevice(m.device), "cudaSetDevice");
        const size_t NB = N * sizeof(float4);
        cuda_check(cudaMemcpyAsync(m.d_pos[m.cur], pos.data(), NB, cudaMemcpyHostToDevice, m.stream), "restore");
        cuda_check(cudaMemcpyAsync(m.d_prev[m.cur], prev.data(), NB, cudaMemcpyHostToDevice, m.stream), "restore");
        cuda_check(cudaMemcpyAsync(m.d_vel[m.cur], vel.data(), NB, cudaMemcpyHostToDevice, m.stream), "restore");
        cuda_check(cudaMemcpyAsync(m.d_origin[m.cur], o, sizeof(o), cudaMemcpyHostToDevice, m.stream), "restore");
        if (susp)
            cuda_check(cudaMemcpyAsync(m.d_payload[m.cur], &pay, sizeof(pay), cudaMemcpyHostToDevice, m.stream),
                       "restore");
        cuda_check(cudaStreamSynchronize(m.stream), "restore");
        m.pending = pending;
        m.forces_dirty = true;
        m.last_applied = last;
        if (pressure != m.pressure) {
            m.pressure = pressure;
            m.pressure_dirty = true;
        }
        m.accepted = accepted;
        m.time = time;
        m.last_dt = last_dt;
    });
}

}  // extern "C"
