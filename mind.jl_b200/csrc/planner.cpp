/*
 * planner.cpp — host-side build planning of libmindgpu.so: discretization of a cell's
 * sections into the cable node tree (mind_discretize, include/mindgpu.h).
 *
 * It restates MIND.jl's discretize (src/model/micro/morphology.jl:406-484) and its
 * geometry integration (src/model/micro/utils/morphology.jl:28-63, section order :77-104):
 *   - sections are visited parents first, each parent chain resolved in input order;
 *   - a root section gets a root node (area 100 um2, no capacitance, no axial);
 *   - each section gets nseg segment nodes whose area, axial conductance to the previous
 *     node and capacitance integrate the geometry over the two half segments around the
 *     segment centre, walking the pt3d spans (a section given by length and diameter is
 *     one span of constant diameter), and one zero-capacitance node at its x = 1 end;
 *   - a section attaches at parent_x of its parent: x = 0 the parent's start, x = 1 its
 *     end, otherwise the segment containing x.
 * The coefficients feed an FP64 solve compared bit for bit with MIND.jl's, so every
 * floating-point operation follows the reference's order (compiled with
 * -ffp-contract=off: nothing is contracted into fused multiply-adds).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mindgpu.h"

namespace {

constexpr double kPi = 3.141592653589793115997963468544185161590576171875;   // the double nearest pi
constexpr double kHalfPi = 0.5 * kPi;

struct Cursor {
    int64_t index;
    double arc, diameter;
};

struct Half {
    double area, resistance, diameter_integral;
};

/* Area, axial resistance and diameter integral from the cursor to `boundary` along the
 * section's samples (utils/morphology.jl:28-63); the cursor moves to the boundary. */
Half integrate(const std::vector<double> &diam, const std::vector<double> &arcs, double boundary, double Ra,
               Cursor &c) {
    double area = 0.0, resistance = 0.0, diameter_integral = 0.0;
    int64_t index = c.index;
    double previous_arc = c.arc, previous_diameter = c.diameter;
    const int64_t last = (int64_t)arcs.size() - 1;
    for (;;) {
        const int64_t next = index + 1;
        const bool at_boundary = arcs[next] > boundary || next == last;
        double arc, diameter;
        if (at_boundary) {
            const double span = arcs[next] - arcs[index];
            const double fraction = std::fabs(span) < 1.0e-10 ? 1.0 : (boundary - arcs[index]) / span;
            arc = boundary;
            diameter = (1.0 - fraction) * diam[index] + fraction * diam[next];
        } else {
            arc = arcs[next];
            diameter = diam[next];
        }
        const double delta = arc - previous_arc;
        diameter_integral += (previous_diameter + diameter) * delta;
        const double distance = delta > 1.0e-15 ? delta : 1.0e-15;
        const double conductance = previous_diameter * diameter / distance;
        resistance += 1.0 / (conductance == 0.0 ? 1.0e-15 : conductance);
        const double jump = diameter - previous_diameter;
        area += (previous_diameter + diameter) * std::sqrt(distance * distance + 0.25 * (jump * jump));
        previous_arc = arc;
        previous_diameter = diameter;
        if (at_boundary) break;
        index = next;
    }
    c = Cursor{index, previous_arc, previous_diameter};
    return Half{kHalfPi * area, ((0.04 * Ra) / kPi) * resistance, 0.5 * diameter_integral};
}

}  // namespace

extern "C" int mind_discretize(const MindSection *sections, int32_t n_sections, int64_t capacity,
                               MindMorphology *out, char *message, int32_t message_len) {
    auto fail = [&](const std::string &why) {
        if (message && message_len > 0) {
            std::strncpy(message, why.c_str(), (size_t)message_len - 1);
            message[message_len - 1] = 0;
        }
        return (int)MIND_ELAYOUT;
    };
    if (!out || n_sections < 0 || (n_sections > 0 && !sections)) {
        fail("invalid arguments");
        return (int)MIND_EARG;
    }
    const int32_t n = n_sections;
    // ---- order: parents before children, each parent chain resolved in input order
    std::vector<int32_t> marks(n, 0), order, pending;
    order.reserve(n);
    for (int32_t start = 0; start < n; ++start) {
        int32_t index = start;
        while (marks[index] != 2) {
            if (marks[index] == 1) return fail("morphology contains a cycle");
            marks[index] = 1;
            pending.push_back(index);
            const int32_t parent = sections[index].parent;
            if (parent < 0) break;
            if (parent >= n) return fail("unknown parent section");
            index = parent;
        }
        while (!pending.empty()) {
            index = pending.back();
            pending.pop_back();
            marks[index] = 2;
            order.push_back(index);
        }
    }
    int64_t total = 0;
    for (int32_t i = 0; i < n; ++i) {
        const MindSection &s = sections[i];
        if (!(s.nseg > 0) || !std::isfinite(s.Ra) || !(s.Ra > 0.0) || !std::isfinite(s.cm) || !(s.cm >= 0.0))
            return fail("invalid segmentation or biophysics on section " + std::to_string(i));
        if (s.n_points >= 2 && !s.points) return fail("pt3d samples missing");
        total += (int64_t)s.nseg + 1 + (s.parent < 0 ? 1 : 0);
    }
    out->node_count = total;
    if (total > capacity) return (int)MIND_ECAPACITY;   // the caller sizes the outputs and calls again
    if (total > 0 && (!out->parent || !out->area || !out->diameter || !out->axial || !out->capacitance ||
                      !out->edge_length))
        return fail("missing output arrays");
    // ---- nodes (1-based ids; node id k is output element k - 1)
    int64_t count = 0;
    std::vector<int64_t> start_node(n, 0), end_node(n, 0), first_segment(n, 0);
    auto add = [&](int64_t parent, double a, double d, double g, double c, double span) {
        out->parent[count] = (int32_t)parent;
        out->area[count] = a;
        out->diameter[count] = d;
        out->axial[count] = g;
        out->capacitance[count] = c;
        out->edge_length[count] = span;
        return ++count;
    };
    auto location = [&](int32_t section, double x) -> int64_t {
        if (x == 0.0) return start_node[section];
        if (x == 1.0) return end_node[section];
        const int32_t nseg = sections[section].nseg;
        int64_t index = (int64_t)std::floor(x * (double)nseg);
        if (index > nseg - 1) index = nseg - 1;
        // a section attached by its x = 1 end lists its segments from the far end
        const bool reversed = sections[section].child_x == 1.0;
        return reversed ? first_segment[section] + (nseg - 1 - index) : first_segment[section] + index;
    };
    std::vector<double> diam, arcs;
    for (int32_t index : order) {
        const MindSection &s = sections[index];
        diam.clear();
        arcs.assign(1, 0.0);
        if (s.n_points >= 2) {
            for (int32_t k = 0; k < s.n_points; ++k) diam.push_back(s.points[4 * k + 3]);
            for (int32_t k = 1; k < s.n_points; ++k) {
                const double *l = s.points + 4 * (k - 1), *r = s.points + 4 * k;
                const double dx = r[0] - l[0], dy = r[1] - l[1], dz = r[2] - l[2];
                arcs.push_back(arcs.back() + std::sqrt(dx * dx + dy * dy + dz * dz));
            }
        } else {
            diam.assign(2, s.diameter);
            const double dx = s.length - 0.0, dy = 0.0 - 0.0, dz = 0.0 - 0.0;
            arcs.push_back(0.0 + std::sqrt(dx * dx + dy * dy + dz * dz));
        }
        if (!(arcs.back() > 0.0)) return fail("section " + std::to_string(index) + " has zero arc length");
        int64_t connection;
        if (s.parent < 0) {
            connection = add(0, 100.0, 0.0, 0.0, 0.0, 0.0);
        } else {
            if (!(s.parent_x >= 0.0 && s.parent_x <= 1.0)) return fail("parent_x must be in [0, 1]");
            connection = location(s.parent, s.parent_x);
        }
        const int32_t nseg = s.nseg;
        const double step = arcs.back() / (double)nseg;
        Cursor cursor{0, arcs[0], diam[0]};
        double previous_right = 0.0;
        const int64_t base = count;
        for (int32_t k = 1; k <= nseg; ++k) {
            const double middle = ((double)k - 0.5) * step;
            const double right = (double)k * step;
            const Half l = integrate(diam, arcs, middle, s.Ra, cursor);
            const Half r = integrate(diam, arcs, right, s.Ra, cursor);
            const double node_area = l.area + r.area;
            add(k == 1 ? connection : base + k - 1, node_area, (l.diameter_integral + r.diameter_integral) / step,
                1.0 / (previous_right + l.resistance), s.cm * node_area * 1.0e-5, k == 1 ? 0.5 * step : step);
            previous_right = r.resistance;
        }
        const int64_t endpoint = add(count, 100.0, 0.0, 1.0 / previous_right, 0.0, 0.5 * step);
        first_segment[index] = base + 1;
        const bool reversed = s.child_x == 1.0;
        start_node[index] = reversed ? endpoint : connection;
        end_node[index] = reversed ? connection : endpoint;
        if (out->section_start) out->section_start[index] = start_node[index];
        if (out->section_end) out->section_end[index] = end_node[index];
        if (out->section_first) out->section_first[index] = first_segment[index];
    }
    return count == total ? (int)MIND_OK : fail("node count mismatch");
}
