// libgap_io_pgm.so: a power-grid-model (PGM) JSON reader and result writer behind the
// reference's IO interface (gap::io::IIOModule, include/gap/io/io_interface.h:8-44), exported as
//   extern "C" gap::io::IIOModule* create_pgm_io_module();
//   extern "C" void destroy_pgm_io_module(gap::io::IIOModule*);
// so that a reference-built caller (gap_b200_main here; the reference's gap_main with its
// BackendFactory::create_io_module, src/core/backend_factory.cpp:21-24, pointed at this
// library) reads PGM input into the reference's NetworkData for the GPU backends.
//
// The conversion follows the reference's own reader (src/io/json_io.cpp:113-382) component by
// component -- node, line, transformer, generic_branch, source, sym_load, sym_gen -- with two
// corrections:
//   * load sign: a PGM sym_load's p_specified / q_specified is consumption, so it enters the
//     NetworkData as a negative injection (the reference copies it unsigned,
//     json_io.cpp:195-211, and the Newton solver sums p_specified + j q_specified of every
//     LOADGEN as an injection, cpu_newton_raphson.cpp:361-367); sym_gen stays positive;
//   * bus types: a source's bus is SLACK at u_ref; every other bus is PQ.  The reference makes
//     a bus PV when a LOADGEN has negative p_specified (json_io.cpp:362-367), which with the
//     corrected sign would turn every loaded bus into a PV bus; PGM's sym_gen has no voltage
//     control.
// It also reads the shunt component (g1, b1) as a SHUNT appliance, which the reference's
// reader skips.  write_results writes the node results as a PGM output dataset (u_pu, u in V,
// u_angle in rad per node of the last network read), plus the solver's convergence flag and
// iteration count; the reference leaves write_results unimplemented (json_io.cpp:505-517).
#include <algorithm>
#include <cmath>
#include <complex>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "gap_b200/gap_interfaces.hpp"
#include "json_min.hpp"

namespace gapb200 {

using json::Json;

namespace {

std::string read_file(std::string const& filename) {
    std::ifstream in(filename, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot open file: " + filename);
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

const Json& component(Json const& data, const char* name) {
    static const Json empty = [] {
        Json j;
        j.kind = Json::Kind::Array;
        return j;
    }();
    const Json* c = data.get(name);
    if (!c || c->kind == Json::Kind::Null) return empty;
    if (!c->is_array()) throw std::runtime_error(std::string("PGM component '") + name + "' is not a list");
    return *c;
}

int8_t status_of(Json const& e, const char* key) {
    return static_cast<int8_t>(e.number(key, 1.0) != 0.0 ? 1 : 0);
}

// line (json_io.cpp:31-66): b1 = 2 pi 50 c1, g1 = b1 tan1 (BranchData::
// set_from_pgm_capacitive_params); i_n default 1 kA
gap::BranchData line(Json const& e) {
    gap::BranchData b;
    b.id = static_cast<int>(e.required("id"));
    b.from_bus = static_cast<int>(e.required("from_node"));
    b.to_bus = static_cast<int>(e.required("to_node"));
    b.from_status = status_of(e, "from_status");
    b.to_status = status_of(e, "to_status");
    b.status = (b.from_status && b.to_status) ? 1 : 0;
    b.branch_type = gap::BranchType::LINE;
    b.r1 = e.required("r1");
    b.x1 = e.required("x1");
    const double c1 = e.number("c1", 0.0), tan1 = e.number("tan1", 0.0);
    b.b1 = c1 > 0.0 ? 2.0 * M_PI * 50.0 * c1 : 0.0;
    b.g1 = b.b1 * tan1;
    b.k = 1.0;
    b.theta = 0.0;
    b.sn = 0.0;
    b.i_n = e.number("i_n", 1000.0);
    return b;
}

// transformer (json_io.cpp:216-268): impedance on the primary base split by the X/R ratio,
// k = u1 / u2 scaled by the tap position, theta = clock x 30 degrees
gap::BranchData transformer(Json const& e) {
    gap::BranchData b;
    b.id = static_cast<int>(e.required("id"));
    b.from_bus = static_cast<int>(e.required("from_node"));
    b.to_bus = static_cast<int>(e.required("to_node"));
    b.from_status = status_of(e, "from_status");
    b.to_status = status_of(e, "to_status");
    b.status = (b.from_status && b.to_status) ? 1 : 0;
    b.branch_type = gap::BranchType::TRAFO;
    const double u1 = e.required("u1"), u2 = e.required("u2"), sn = e.required("sn"),
                 uk = e.required("uk");
    const double z = uk * (u1 * u1) / sn;
    const double xr = e.has("rx_ratio") ? 1.0 / e.required("rx_ratio") : 10.0;
    const double rf = 1.0 / std::sqrt(1.0 + xr * xr);
    b.r1 = z * rf;
    b.x1 = z * xr * rf;
    b.k = u1 / u2;
    if (e.has("tap_pos") && e.has("tap_size"))
        b.k *= 1.0 + e.required("tap_pos") * e.required("tap_size") / 100000.0;
    b.theta = e.has("clock") ? e.required("clock") * M_PI / 6.0 : 0.0;
    b.sn = sn;
    b.i_n = sn / (std::sqrt(3.0) * std::min(u1, u2));
    b.g1 = 0.0;
    b.b1 = 0.0;
    return b;
}

// generic_branch (json_io.cpp:273-309)
gap::BranchData generic_branch(Json const& e) {
    gap::BranchData b;
    b.id = static_cast<int>(e.required("id"));
    b.from_bus = static_cast<int>(e.required("from_node"));
    b.to_bus = static_cast<int>(e.required("to_node"));
    b.from_status = status_of(e, "from_status");
    b.to_status = status_of(e, "to_status");
    b.status = (b.from_status && b.to_status) ? 1 : 0;
    b.branch_type = gap::BranchType::GENERIC;
    b.r1 = e.required("r1");
    b.x1 = e.required("x1");
    b.g1 = e.number("g1", 0.0);
    b.b1 = e.number("b1", 0.0);
    b.k = e.number("k", 1.0);
    b.theta = e.number("shift", 0.0);
    b.sn = e.number("sn", 0.0);
    if (e.has("i_n"))
        b.i_n = e.required("i_n");
    else if (b.sn > 0.0)
        b.i_n = b.sn / (std::sqrt(3.0) * 20000.0);
    return b;
}

gap::ApplianceData appliance(Json const& e, gap::ApplianceType type) {
    gap::ApplianceData a;
    a.id = static_cast<int>(e.required("id"));
    a.node = static_cast<int>(e.required("node"));
    a.status = status_of(e, "status");
    a.type = type;
    return a;
}

}  // namespace

class PgmIOModule final : public gap::io::IIOModule {
  public:
    gap::NetworkData read_network_data(std::string const& filename) override {
        const Json root = json::parse(read_file(filename));
        if (!root.is_object()) throw std::runtime_error("PGM input: the document is not an object");
        gap::NetworkData net;
        if (const Json* v = root.get("version"); v && v->kind == Json::Kind::String) net.version = v->str;
        if (const Json* v = root.get("type"); v && v->kind == Json::Kind::String) net.type = v->str;
        if (const Json* v = root.get("is_batch"); v && v->kind == Json::Kind::Bool) net.is_batch = v->b;
        const Json* data = root.get("data");
        if (!data || !data->is_object()) throw std::runtime_error("PGM input: 'data' object missing");
        for (Json const& e : component(*data, "node").arr) {
            gap::BusData b;
            b.id = static_cast<int>(e.required("id"));
            b.u_rated = e.required("u_rated");
            b.bus_type = gap::BusType::PQ;
            b.energized = 0;
            b.u = b.u_rated;
            b.u_pu = 1.0;
            b.u_angle = 0.0;
            net.buses.push_back(b);
        }
        for (Json const& e : component(*data, "line").arr) net.branches.push_back(line(e));
        for (Json const& e : component(*data, "transformer").arr) net.branches.push_back(transformer(e));
        for (Json const& e : component(*data, "generic_branch").arr)
            net.branches.push_back(generic_branch(e));
        std::unordered_map<int, double> u_ref;  // node -> u_ref of its (last) active source
        for (Json const& e : component(*data, "source").arr) {
            gap::ApplianceData a = appliance(e, gap::ApplianceType::SOURCE);
            a.u_ref = e.number("u_ref", 1.0);
            a.u_ref_angle = e.number("u_ref_angle", 0.0);
            a.sk = e.number("sk", 1e10);
            a.rx_ratio = e.number("rx_ratio", 0.1);
            if (a.status) u_ref[a.node] = a.u_ref;
            net.appliances.push_back(a);
        }
        for (Json const& e : component(*data, "sym_load").arr) {
            gap::ApplianceData a = appliance(e, gap::ApplianceType::LOADGEN);
            a.p_specified = -e.number("p_specified", 0.0);  // consumption -> injection
            a.q_specified = -e.number("q_specified", 0.0);
            net.appliances.push_back(a);
        }
        for (Json const& e : component(*data, "sym_gen").arr) {
            gap::ApplianceData a = appliance(e, gap::ApplianceType::LOADGEN);
            a.p_specified = e.number("p_specified", 0.0);
            a.q_specified = e.number("q_specified", 0.0);
            net.appliances.push_back(a);
        }
        for (Json const& e : component(*data, "shunt").arr) {
            gap::ApplianceData a = appliance(e, gap::ApplianceType::SHUNT);
            a.g1 = e.number("g1", 0.0);
            a.b1 = e.number("b1", 0.0);
            net.appliances.push_back(a);
        }
        for (auto& b : net.buses) {
            auto it = u_ref.find(b.id);
            if (it != u_ref.end()) {
                b.bus_type = gap::BusType::SLACK;
                if (it->second > 0.0) b.u_pu = it->second;
            }
        }
        net.num_buses = static_cast<int>(net.buses.size());
        net.num_branches = static_cast<int>(net.branches.size());
        net.num_appliances = static_cast<int>(net.appliances.size());
        ids_.clear();
        u_rated_.clear();
        for (auto const& b : net.buses) {
            ids_.push_back(b.id);
            u_rated_.push_back(b.u_rated);
        }
        return net;
    }

    void write_results(std::string const& filename, gap::ComplexVector const& v, bool converged,
                       int iterations) override {
        std::ofstream out(filename);
        if (!out) throw std::runtime_error("Cannot open file: " + filename);
        out << "{\n  \"version\": \"1.0\",\n  \"type\": \"sym_output\",\n  \"is_batch\": false,\n"
            << "  \"attributes\": {},\n  \"converged\": " << (converged ? "true" : "false")
            << ",\n  \"iterations\": " << iterations << ",\n  \"data\": {\n    \"node\": [";
        for (size_t i = 0; i < v.size(); ++i) {
            const double m = std::abs(v[i]);
            const bool known = i < ids_.size();
            out << (i ? "," : "") << "\n      {\"id\": " << (known ? ids_[i] : static_cast<int>(i))
                << ", \"energized\": 1, \"u_pu\": " << json::number(m) << ", \"u\": "
                << json::number(known ? m * u_rated_[i] : m) << ", \"u_angle\": "
                << json::number(std::arg(v[i])) << "}";
        }
        out << "\n    ]\n  }\n}\n";
        if (!out) throw std::runtime_error("write failed: " + filename);
    }

    bool validate_input_format(std::string const& filename) override {
        try {
            const Json root = json::parse(read_file(filename));
            const Json* data = root.get("data");
            if (!data || !data->is_object()) return false;
            const Json* nodes = data->get("node");
            if (!nodes || !nodes->is_array() || nodes->arr.empty()) return false;
            for (Json const& e : nodes->arr)
                if (!e.get("id") || !e.get("u_rated")) return false;
            return true;
        } catch (std::exception const&) {
            return false;
        }
    }

  private:
    std::vector<int> ids_;          // bus ids of the last network read, in bus order
    std::vector<double> u_rated_;   // and their rated voltages (V)
};

}  // namespace gapb200

extern "C" {
gap::io::IIOModule* create_pgm_io_module() { return new gapb200::PgmIOModule(); }
void destroy_pgm_io_module(gap::io::IIOModule* m) { delete m; }
}
