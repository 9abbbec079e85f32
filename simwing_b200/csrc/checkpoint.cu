// Structure::checkpoint / restore (src/fsi/structure.cpp:961-1027) for the
// device state: an opaque, checksummed little-endian byte image bound to the
// definition fingerprint.  Restoring an image taken from the same structure
// reproduces its state bit for bit (positions are stored as the frame
// origin plus the FP32 offsets, both exactly).  With fabric self-contact the
// image also holds the contact multiplier table (the warm starts and the
// record book that carry from step to step, as SoftBodyCheckpoint::State
// holds contactMultipliers and contactRecords) and the contact diagnostics.
#include "structure_impl.h"

#include <cmath>
#include <cstring>

namespace swb {
namespace {

constexpr char kMagic[8] = {'S', 'W', 'B', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kVersion = 2;

// One multiplier table entry in the image: code, lambda, normal, flags.
constexpr uint64_t kEntryBytes = 8 + 8 + 24 + 4;
constexpr uint64_t kContactDiagBytes = 8 + 8 + 8 + 8;

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

// The committed multiplier table of a contact structure (the entries of the
// current ping-pong buffer, in code order) and its contact diagnostics.
struct ContactImage {
    std::vector<ContactEntry> entries;
    ContactDiagDev diag{};
};

ContactImage fetch_contact(const StructureImpl& m) {
    ContactImage c;
    uint32_t meta[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(meta, m.contact_host.table_meta, sizeof(meta), cudaMemcpyDeviceToHost, m.stream),
               "read");
    cuda_check(cudaStreamSynchronize(m.stream), "read");
    if (meta[0] > 1u || meta[1] > m.contact_host.table_cap)
        raise(SWB_CUDA_ERROR, "internal error: contact table state out of range");
    c.entries.resize(meta[1]);
    if (meta[1])
        cuda_check(cudaMemcpyAsync(c.entries.data(), m.contact_host.table[meta[0]],
                                   meta[1] * sizeof(ContactEntry), cudaMemcpyDeviceToHost, m.stream), "read");
    cuda_check(cudaMemcpyAsync(&c.diag, m.d_cdiag[m.cur], sizeof(c.diag), cudaMemcpyDeviceToHost, m.stream), "read");
    cuda_check(cudaStreamSynchronize(m.stream), "read");
    return c;
}

uint64_t image_bytes(const StructureImpl& m, uint64_t contact_entries) {
    const uint64_t N = m.def.nodes.size();
    uint64_t bytes = 8 + 4 + 4 + 4 + 4 + 8 + 8 + 8 + 8 + 24 + 8 + N * 72 + N * 24 + 24 + 8 + m.pressure.size() * 8 +
                     (m.def.has_suspension ? sizeof(DevPayloadState) : 0) + 8;
    if (m.d_contact) bytes += 8 + contact_entries * kEntryBytes + kContactDiagBytes;
    return bytes;
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
    w.u32(m.d_contact ? 1u : 0u);
    w.u32(0u);
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
    if (m.d_contact) {
        const ContactImage c = fetch_contact(m);
        w.u64(c.entries.size());
        for (const ContactEntry& e : c.entries) {
            w.u64(e.code);
            w.f64(e.lambda);
            w.f64(e.normal[0]); w.f64(e.normal[1]); w.f64(e.normal[2]);
            w.u32(e.flags);
        }
        w.u64(c.diag.candidates);
        w.u64(c.diag.active);
        w.u64(c.diag.records);
        w.f64(c.diag.max_penetration);
    }
    const uint64_t sum = fnv1a(w.bytes.data(), w.bytes.size());
    w.u64(sum);
    return w.bytes;
}

bool is_finite_value(double v) { return std::isfinite(v); }

// A restored pilot state must be one the solver can have written: every
// field finite, a unit orientation quaternion (FP32 normalised) and a
// non-negative residual.
void check_payload(const DevPayloadState& p) {
    const float* f = reinterpret_cast<const float*>(&p);
    for (size_t i = 0; i < sizeof(p) / sizeof(float); ++i)
        if (!std::isfinite(f[i])) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: non-finite pilot state");
    const double qq = double(p.q.x) * p.q.x + double(p.q.y) * p.q.y + double(p.q.z) * p.q.z + double(p.q.w) * p.q.w;
    if (!(std::fabs(qq - 1.0) <= 1.0e-4))
        raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: pilot orientation is not a unit quaternion");
    if (!(p.max_residual >= 0.0f)) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: pilot residual");
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

swb_status swb_structure_checkpoint_size(const swb_structure* s, uint64_t* bytes) {
    return guarded([&] {
        if (!s || !bytes) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        uint64_t entries = 0;
        if (m.d_contact) entries = fetch_contact(m).entries.size();
        *bytes = image_bytes(m, entries);
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
        const bool contact = r.u32() != 0;
        if (r.u32() != 0u) raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
        if (r.u64() != m.fingerprint)
            raise(SWB_INVALID_ARGUMENT, "Structure checkpoint belongs to a different definition");
        if (susp != m.def.has_suspension || contact != (m.d_contact != nullptr))
            raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint");
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
        if (susp) {
            r.raw(&pay, sizeof(pay));
            check_payload(pay);
        }
        ContactImage cimg;
        if (contact) {
            const uint64_t n = r.u64();
            if (n > m.contact_host.table_cap || n * kEntryBytes > r.n - r.at)
                raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: contact table");
            cimg.entries.resize(n);
            for (uint64_t k = 0; k < n; ++k) {
                ContactEntry& e = cimg.entries[k];
                std::memset(&e, 0, sizeof e);
                e.code = r.u64();
                e.lambda = r.f64();
                e.normal[0] = r.f64(); e.normal[1] = r.f64(); e.normal[2] = r.f64();
                e.flags = r.u32();
                // entries are sorted by code, with finite values and known flags
                if ((k && !(cimg.entries[k - 1].code < e.code)) || !is_finite_value(e.lambda) ||
                    !is_finite_value(e.normal[0]) || !is_finite_value(e.normal[1]) || !is_finite_value(e.normal[2]) ||
                    (e.flags & ~uint32_t(kEntryApplied | kEntryRecord | kEntryVisited)) != 0u)
                    raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: contact table");
            }
            cimg.diag.candidates = r.u64();
            cimg.diag.active = r.u64();
            cimg.diag.records = r.u64();
            cimg.diag.max_penetration = r.f64();
            if (!is_finite_value(cimg.diag.max_penetration) || cimg.diag.active > cimg.diag.records)
                raise(SWB_INVALID_ARGUMENT, "Invalid structure checkpoint: contact diagnostics");
        }
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
        if (contact) {
            const uint32_t meta[2] = {0u, static_cast<uint32_t>(cimg.entries.size())};
            if (!cimg.entries.empty())
                cuda_check(cudaMemcpyAsync(m.contact_host.table[0], cimg.entries.data(),
                                           cimg.entries.size() * sizeof(ContactEntry), cudaMemcpyHostToDevice,
                                           m.stream), "restore");
            cuda_check(cudaMemcpyAsync(m.contact_host.table_meta, meta, sizeof(meta), cudaMemcpyHostToDevice,
                                       m.stream), "restore");
            cuda_check(cudaMemcpyAsync(m.d_cdiag[m.cur], &cimg.diag, sizeof(cimg.diag), cudaMemcpyHostToDevice,
                                       m.stream), "restore");
        }
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
