// Pneumatic port mass flows: the orifice and linear-conductance laws of
// softwing's cell-air model (pneumatics.cpp:112-232), one device thread per
// port.
//
// Each thread follows the reference's order of operations.  The conductance
// law is plain arithmetic and matches the reference bit for bit (this
// translation unit is built without FMA contraction).  The orifice law
// calls pow, and CUDA's double pow and the host C library's may differ in
// the last bits, so orifice flows agree to a few ulp.  Every refusal of the
// reference (AirProperties::validate, validateFlowState, validateOpening,
// the port constants, a non-finite flow) is decided on the device per port;
// the host reports the first refusing port.
#include "simwing_b200.h"

#include "common.h"
#include "structure_impl.h"

#include <algorithm>
#include <cstdint>
#include <vector>

namespace swb {
namespace {

__device__ __forceinline__ bool finite_positive(double v) { return v > 0.0 && isfinite(v); }

__device__ __forceinline__ bool valid_state(const swb_flow_zone_state& s) {
    return finite_positive(s.absolute_pressure) && finite_positive(s.absolute_temperature);
}

__device__ __forceinline__ bool valid_opening(double o) { return isfinite(o) && !(o < 0.0) && !(o > 1.0); }

// evaluateOrificeMassFlow (pneumatics.cpp:132-197).  Returns false where the
// reference throws.
__device__ bool orifice_flow(const swb_flow_zone_state& first, const swb_flow_zone_state& second,
                             const swb_air_properties& air, const swb_port_def& port, swb_mass_flow& r) {
    if (!finite_positive(air.specific_gas_constant) || !(air.heat_capacity_ratio > 1.0) ||
        !isfinite(air.heat_capacity_ratio))
        return false;
    if (!valid_state(first) || !valid_state(second) || !valid_opening(port.opening_fraction)) return false;
    if (!(port.discharge_coefficient > 0.0) || port.discharge_coefficient > 1.0 ||
        !isfinite(port.discharge_coefficient) || !finite_positive(port.effective_area))
        return false;
    const double gamma = air.heat_capacity_ratio;
    r.critical_pressure_ratio = pow(2.0 / (gamma + 1.0), gamma / (gamma - 1.0));
    if (first.absolute_pressure == second.absolute_pressure || port.opening_fraction == 0.0) return true;

    const bool first_upstream = first.absolute_pressure > second.absolute_pressure;
    const swb_flow_zone_state& up = first_upstream ? first : second;
    const swb_flow_zone_state& down = first_upstream ? second : first;
    r.direction = first_upstream ? SWB_FLOW_FIRST_TO_SECOND : SWB_FLOW_SECOND_TO_FIRST;
    const double ratio = down.absolute_pressure / up.absolute_pressure;
    r.pressure_ratio = ratio < 0.0 ? 0.0 : (1.0 < ratio ? 1.0 : ratio);

    const double scale = up.absolute_pressure / sqrt(air.specific_gas_constant * up.absolute_temperature);
    double flux;
    if (r.pressure_ratio <= r.critical_pressure_ratio) {
        r.choked = 1u;
        flux = scale * sqrt(gamma) * pow(2.0 / (gamma + 1.0), (gamma + 1.0) / (2.0 * (gamma - 1.0)));
    } else {
        const double first_power = pow(r.pressure_ratio, 2.0 / gamma);
        const double second_power = pow(r.pressure_ratio, (gamma + 1.0) / gamma);
        const double x = (2.0 * gamma / (gamma - 1.0)) * (first_power - second_power);
        const double radicand = 0.0 < x ? x : 0.0;  // std::max(0.0, x)
        flux = scale * sqrt(radicand);
    }
    r.magnitude = port.discharge_coefficient * port.effective_area * port.opening_fraction * flux;
    if (!isfinite(r.magnitude)) return false;
    r.signed_mass_rate = first_upstream ? r.magnitude : -r.magnitude;
    return true;
}

// evaluateConductanceMassFlow (pneumatics.cpp:199-232).
__device__ bool conductance_flow(const swb_flow_zone_state& first, const swb_flow_zone_state& second,
                                 const swb_port_def& port, swb_mass_flow& r) {
    if (!valid_state(first) || !valid_state(second) || !valid_opening(port.opening_fraction)) return false;
    if (!finite_positive(port.mass_conductance)) return false;
    if (first.absolute_pressure == second.absolute_pressure || port.opening_fraction == 0.0) return true;
    r.signed_mass_rate =
        port.mass_conductance * port.opening_fraction * (first.absolute_pressure - second.absolute_pressure);
    r.magnitude = fabs(r.signed_mass_rate);
    r.direction = r.signed_mass_rate > 0.0 ? SWB_FLOW_FIRST_TO_SECOND : SWB_FLOW_SECOND_TO_FIRST;
    const double a = first.absolute_pressure, b = second.absolute_pressure;
    const double high = a < b ? b : a;  // std::max
    const double low = b < a ? b : a;   // std::min
    r.pressure_ratio = low / high;
    return isfinite(r.signed_mass_rate);
}

// `zone_count`: ports naming a zone past it are refused (the host entry
// point rejects them before the launch; the device-array form has no host
// copy of the ports to check).
__global__ void port_flow_kernel(swb_air_properties air, const swb_flow_zone_state* __restrict__ zones,
                                 uint64_t zone_count, const swb_port_def* __restrict__ ports, uint64_t count,
                                 swb_mass_flow* out, unsigned long long* failed) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    const swb_port_def port = ports[i];
    swb_mass_flow r{};  // MassFlowEvaluation's defaults
    r.pressure_ratio = 1.0;
    r.critical_pressure_ratio = 1.0;
    bool ok = false;
    if (port.reserved == 0u && port.first < zone_count && port.second < zone_count) {
        const swb_flow_zone_state first = zones[port.first], second = zones[port.second];
        if (port.kind == SWB_PORT_ORIFICE) ok = orifice_flow(first, second, air, port, r);
        else if (port.kind == SWB_PORT_CONDUCTANCE) ok = conductance_flow(first, second, port, r);
    }
    out[i] = r;
    if (!ok) atomicMin(failed, static_cast<unsigned long long>(i));
}

__global__ void set_word(unsigned long long* word, unsigned long long value) { *word = value; }

template <class T>
struct Scratch {
    T* ptr = nullptr;
    explicit Scratch(uint64_t n) { cuda_check(cudaMalloc(&ptr, std::max<uint64_t>(n, 1) * sizeof(T)), "cudaMalloc (port flows)"); }
    ~Scratch() { cudaFree(ptr); }
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
};

}  // namespace
}  // namespace swb

using namespace swb;

swb_status swb_port_mass_flows(const swb_air_properties* air, const swb_flow_zone_state* zones, uint64_t zone_count,
                               const swb_port_def* ports, uint64_t port_count, swb_mass_flow* out,
                               uint64_t* failed_port) {
    return guarded([&] {
        if (failed_port) *failed_port = port_count;
        if (!air || (port_count && (!ports || !out || !zones))) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!port_count) return;
        for (uint64_t i = 0; i < port_count; ++i)
            if (ports[i].first >= zone_count || ports[i].second >= zone_count)
                raise(SWB_OUT_OF_RANGE, "pneumatic port references an unknown zone");
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
            raise(SWB_CUDA_ERROR, "no CUDA device: the port flow kernel needs a GPU");
        Scratch<swb_flow_zone_state> d_zones(zone_count);
        Scratch<swb_port_def> d_ports(port_count);
        Scratch<swb_mass_flow> d_out(port_count);
        Scratch<unsigned long long> d_failed(1);
        const unsigned long long none = port_count;
        cuda_check(cudaMemcpy(d_zones.ptr, zones, zone_count * sizeof(swb_flow_zone_state), cudaMemcpyHostToDevice),
                   "upload zones");
        cuda_check(cudaMemcpy(d_ports.ptr, ports, port_count * sizeof(swb_port_def), cudaMemcpyHostToDevice),
                   "upload ports");
        cuda_check(cudaMemcpy(d_failed.ptr, &none, sizeof none, cudaMemcpyHostToDevice), "upload");
        port_flow_kernel<<<static_cast<unsigned>((port_count + 255) / 256), 256>>>(
            *air, d_zones.ptr, zone_count, d_ports.ptr, port_count, d_out.ptr, d_failed.ptr);
        cuda_check(cudaGetLastError(), "port_flow_kernel");
        unsigned long long failed = none;
        cuda_check(cudaMemcpy(&failed, d_failed.ptr, sizeof failed, cudaMemcpyDeviceToHost), "download");
        cuda_check(cudaMemcpy(out, d_out.ptr, port_count * sizeof(swb_mass_flow), cudaMemcpyDeviceToHost),
                   "download flows");
        if (failed != none) {
            if (failed_port) *failed_port = failed;
            raise(SWB_INVALID_ARGUMENT, "pneumatic port flow refused (invalid air, zone state, opening, port "
                                        "constants or a non-finite flow)");
        }
    });
}

swb_status swb_port_mass_flows_device(const swb_air_properties* air, const swb_flow_zone_state* zones,
                                      uint64_t zone_count, const swb_port_def* ports, uint64_t port_count,
                                      swb_mass_flow* out, uint64_t* failed_port, void* stream) {
    return guarded([&] {
        if (!air || !failed_port || (port_count && (!ports || !out || !zones)))
            raise(SWB_INVALID_ARGUMENT, "null argument");
        static_assert(sizeof(uint64_t) == sizeof(unsigned long long), "64-bit word");
        auto* failed = reinterpret_cast<unsigned long long*>(failed_port);
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        set_word<<<1, 1, 0, s>>>(failed, port_count);
        cuda_check(cudaGetLastError(), "set_word");
        if (!port_count) return;
        port_flow_kernel<<<static_cast<unsigned>((port_count + 255) / 256), 256, 0, s>>>(
            *air, zones, zone_count, ports, port_count, out, failed);
        cuda_check(cudaGetLastError(), "port_flow_kernel");
    });
}
