// Internal host-side declarations shared by the library's translation units.
#pragma once

#include "simwing_b200.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace swb {

// Error carrying an swb_status; every C-ABI entry point catches it and
// stores the message for swb_last_error() and, when the failure has one,
// its detail (suspension phase and entity, contact feature key) for
// swb_last_error_detail().
struct Error : std::runtime_error {
    swb_status status;
    bool has_detail = false;
    swb_error_detail detail{};
    Error(swb_status s, const std::string& message)
        : std::runtime_error(message), status(s) {}
    Error(swb_status s, const std::string& message, const swb_error_detail& d)
        : std::runtime_error(message), status(s), has_detail(true), detail(d) {
        detail.status = static_cast<uint32_t>(s);
    }
};

[[noreturn]] inline void raise(swb_status status, const std::string& message) {
    throw Error(status, message);
}

void set_last_error(const std::string& message);
void set_last_error_detail(const swb_error_detail* detail);  // nullptr clears it

// Runs `body` and converts exceptions into a status + thread-local message.
template <class F>
swb_status guarded(F&& body) {
    try {
        body();
        return SWB_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        set_last_error_detail(e.has_detail ? &e.detail : nullptr);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("out of host memory");
        return SWB_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return SWB_INVALID_ARGUMENT;
    } catch (...) {
        set_last_error("unknown exception");
        return SWB_INVALID_ARGUMENT;
    }
}

// Owned copy of a swb_structure_definition.  `view` points into the
// vectors and is refreshed by sync_view().
struct OwnedDefinition {
    std::vector<swb_node_def> nodes;
    std::vector<swb_triangle_def> triangles;
    std::vector<swb_constraint_def> constraints;
    std::vector<swb_membrane_def> membranes;
    std::vector<swb_dihedral_def> dihedrals;
    bool has_contact = false;
    swb_fabric_contact_def contact{};
    bool has_suspension = false;
    swb_suspension_def suspension{};
    std::vector<swb_suspension_attachment> attachments;
    std::vector<swb_suspension_junction> junctions;
    std::vector<swb_pilot_harness> harness;
    std::vector<swb_suspension_segment> segments;
    swb_structure_definition view{};

    void assign(const swb_structure_definition& source);
    void sync_view();
};

void validate_definition(const swb_structure_definition& d);
uint64_t definition_fingerprint(const swb_structure_definition& d);

// Reference greedy line-graph colouring (soft_body.cpp:1978-2075).
struct ReferenceColouring {
    std::vector<uint64_t> order;
    std::vector<uint64_t> offsets;
    uint64_t parallel_colours = 0;
};
ReferenceColouring reference_colouring(uint64_t node_count,
                                       const std::vector<uint32_t>& a,
                                       const std::vector<uint32_t>& b);

}  // namespace swb

struct swb_definition {
    swb::OwnedDefinition def;
};
