// lrt_host.cpp — host-side scene assembly for liblrt (compiled with -ffp-contract=off so every float
// operation rounds as the reference's host code does).
#include "lrt_host.h"

#include <math.h>
#include <cmath>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <thread>
#include <utility>

#include "lrt_math.cuh"

namespace lrt {

namespace {

// ------------------------------------------------------------------------------------------------
// SAH kd-tree (same algorithm and constants as src/accelerator/sah_kdtree.h:141-347)

constexpr float kTraversalCost = 15.0f;
constexpr float kQueryCost = 20.0f;
constexpr float kEmptySpaceBonus = 0.9f;
constexpr int kStopPrims = 6;
constexpr int kMaxBadRefines = 3;

struct Box {
    f3 lo{kInfHost(), kInfHost(), kInfHost()};
    f3 hi{-kInfHost(), -kInfHost(), -kInfHost()};
    static float kInfHost() { return std::numeric_limits<float>::infinity(); }
    void extend(f3 p) {  // aabb::extend(point), aabb.h:9-16
        lo = f3{smin(lo.x, p.x), smin(lo.y, p.y), smin(lo.z, p.z)};
        hi = f3{smax(hi.x, p.x), smax(hi.y, p.y), smax(hi.z, p.z)};
    }
    void extend(const Box& b) {
        extend(b.lo);
        extend(b.hi);
    }
    float surface_area() const {  // aabb.h:24-27
        const f3 e = hi - lo;
        return 2.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
    }
    float lo_a(int a) const { return comp(lo, a); }
    float hi_a(int a) const { return comp(hi, a); }
    void set_lo(int a, float v) { (a == 0 ? lo.x : (a == 1 ? lo.y : lo.z)) = v; }
    void set_hi(int a, float v) { (a == 0 ? hi.x : (a == 1 ? hi.y : hi.z)) = v; }
};

struct Event {
    float position;
    uint32_t index;
    uint8_t type;  // 0 end, 1 planar, 2 start
    uint8_t axis;
};

struct RawNode {
    bool leaf = false;
    int axis = 0;
    float split = 0.0f;
    int left = -1;
    int right = -1;
    int first = 0;
    int count = 0;
};

class KdBuilder {
public:
    KdBuilder(const float* bmin, const float* bmax, uint32_t count) : bmin_(bmin), bmax_(bmax), side_(count, 0) {}

    void run(uint32_t count) {
        if(count == 0) return;
        Box root;
        for(uint32_t i = 0; i < count; ++i) {
            Box b;
            b.lo = load3(bmin_ + 3 * i);
            b.hi = load3(bmax_ + 3 * i);
            root.extend(b);
        }
        std::vector<uint32_t> prims(count);
        for(uint32_t i = 0; i < count; ++i) prims[i] = i;
        const int depth_limit = std::min(48, static_cast<int>(8.0f + 1.3f * log2f(static_cast<float>(count))));
        max_depth_ = std::max(depth_limit, 1);
        // The events are sorted once here. A child's events are its primitives' unclipped boxes, so they
        // are a subsequence of its parent's sorted list: filtering keeps them sorted, and every node sees
        // the list it would have sorted itself (the reference sorts per node, sah_kdtree.h:196-231).
        std::vector<Event> events;
        events.reserve(static_cast<size_t>(count) * 6);
        for(const uint32_t prim : prims) {
            for(uint8_t axis = 0; axis < 3; ++axis) {
                const float lo = bmin_[3 * prim + axis];
                const float hi = bmax_[3 * prim + axis];
                if(lo == hi) {
                    events.push_back(Event{lo, prim, 1, axis});
                } else {
                    events.push_back(Event{lo, prim, 2, axis});
                    events.push_back(Event{hi, prim, 0, axis});
                }
            }
        }
        // keys (axis, position, type, index) are unique per event, so the order is fully determined
        std::sort(events.begin(), events.end(), [](const Event& a, const Event& b) {
            if(a.axis != b.axis) return a.axis < b.axis;
            if(a.position != b.position) return a.position < b.position;
            if(a.type != b.type) return a.type < b.type;
            return a.index < b.index;
        });
        build(prims, events, root, 1, 0);
    }

    std::vector<RawNode> nodes;
    std::vector<uint32_t> ordered;

private:
    std::pair<float, float> split_probability(const Box& box, int axis, float left_width, float right_width) const {
        const f3 edge = box.hi - box.lo;
        const float denom = edge.x * edge.y + edge.y * edge.z + edge.x * edge.z;
        const float temp = 1.0f / denom;
        float face, perimeter;
        if(axis == 0) {
            face = edge.y * edge.z;
            perimeter = edge.y + edge.z;
        } else if(axis == 1) {
            face = edge.x * edge.z;
            perimeter = edge.x + edge.z;
        } else {
            face = edge.x * edge.y;
            perimeter = edge.x + edge.y;
        }
        return {(face + perimeter * left_width) * temp, (face + perimeter * right_width) * temp};
    }

    void make_leaf(int index, const std::vector<uint32_t>& prims) {
        nodes[index].leaf = true;
        nodes[index].first = static_cast<int>(ordered.size());
        nodes[index].count = static_cast<int>(prims.size());
        ordered.insert(ordered.end(), prims.begin(), prims.end());
    }

    // events: the sorted events of `prims` (released once the children's lists are made)
    float build(const std::vector<uint32_t>& prims, std::vector<Event>& events, const Box& voxel, int depth,
                int bad_refines) {
        const int index = static_cast<int>(nodes.size());
        nodes.emplace_back();
        const int prim_count = static_cast<int>(prims.size());
        const float leaf_cost = static_cast<float>(prim_count) * kQueryCost;
        if(prim_count <= kStopPrims || depth >= max_depth_ || voxel.surface_area() <= 0.0f) {
            make_leaf(index, prims);
            return leaf_cost;
        }

        int num_left[3] = {0, 0, 0};
        int num_right[3] = {prim_count, prim_count, prim_count};
        float best_cost = std::numeric_limits<float>::infinity();
        int best_axis = 0;
        float best_position = 0.0f;
        bool planar_left = false;

        const size_t n_events = events.size();
        for(size_t cursor = 0; cursor < n_events;) {
            const int axis = events[cursor].axis;
            const float position = events[cursor].position;
            int num_start = 0, num_end = 0, num_planar = 0;
            while(cursor < n_events && events[cursor].axis == axis && events[cursor].position == position &&
                  events[cursor].type == 0) {
                ++num_end;
                ++cursor;
            }
            while(cursor < n_events && events[cursor].axis == axis && events[cursor].position == position &&
                  events[cursor].type == 1) {
                ++num_planar;
                ++cursor;
            }
            while(cursor < n_events && events[cursor].axis == axis && events[cursor].position == position &&
                  events[cursor].type == 2) {
                ++num_start;
                ++cursor;
            }
            num_right[axis] -= num_planar + num_end;
            if(position > voxel.lo_a(axis) && position < voxel.hi_a(axis)) {
                const auto probability =
                    split_probability(voxel, axis, position - voxel.lo_a(axis), voxel.hi_a(axis) - position);
                const int n_l = num_left[axis];
                const int n_r = num_right[axis];
                if(num_planar == 0) {
                    float cost = kTraversalCost + kQueryCost * (probability.first * static_cast<float>(n_l) +
                                                                probability.second * static_cast<float>(n_r));
                    if(n_l == 0 || n_r == 0) cost *= kEmptySpaceBonus;
                    if(cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_position = position;
                    }
                } else {
                    float cost_left = kTraversalCost + kQueryCost * (probability.first * static_cast<float>(n_l + num_planar) +
                                                                     probability.second * static_cast<float>(n_r));
                    float cost_right = kTraversalCost + kQueryCost * (probability.first * static_cast<float>(n_l) +
                                                                      probability.second * static_cast<float>(n_r + num_planar));
                    if(n_l + num_planar == 0 || n_r == 0) cost_left *= kEmptySpaceBonus;
                    if(n_l == 0 || n_r + num_planar == 0) cost_right *= kEmptySpaceBonus;
                    if(cost_left < best_cost || cost_right < best_cost) {
                        planar_left = cost_left < cost_right;
                        best_cost = planar_left ? cost_left : cost_right;
                        best_axis = axis;
                        best_position = position;
                    }
                }
            }
            num_left[axis] += num_start + num_planar;
        }

        if(best_cost >= leaf_cost) {
            if((best_cost > 4.0f * leaf_cost && prim_count < 16) || bad_refines >= kMaxBadRefines ||
               best_cost == std::numeric_limits<float>::infinity()) {
                make_leaf(index, prims);
                return leaf_cost;
            }
            ++bad_refines;
        }

        // side: 0 both, 1 left only, 2 right only (sah_kdtree.h:290-306); only this node's prims are touched
        for(const uint32_t prim : prims) side_[prim] = 0;
        for(const Event& e : events) {
            if(e.axis != best_axis) continue;
            if(e.type == 0 && e.position <= best_position) {
                side_[e.index] = 1;
            } else if(e.type == 2 && e.position >= best_position) {
                side_[e.index] = 2;
            } else if(e.type == 1) {
                side_[e.index] = (e.position < best_position || (e.position == best_position && planar_left)) ? 1 : 2;
            }
        }
        std::vector<uint32_t> left_prims, right_prims;
        for(const uint32_t prim : prims) {
            if(side_[prim] == 1) {
                left_prims.push_back(prim);
            } else if(side_[prim] == 2) {
                right_prims.push_back(prim);
            } else {
                left_prims.push_back(prim);
                right_prims.push_back(prim);
            }
        }
        std::vector<Event> left_events, right_events;
        left_events.reserve(left_prims.size() * 6);
        right_events.reserve(right_prims.size() * 6);
        for(const Event& e : events) {
            const uint8_t sd = side_[e.index];
            if(sd != 2) left_events.push_back(e);
            if(sd != 1) right_events.push_back(e);
        }
        events.clear();
        events.shrink_to_fit();

        Box left_voxel = voxel;
        Box right_voxel = voxel;
        left_voxel.set_hi(best_axis, best_position);
        right_voxel.set_lo(best_axis, best_position);

        const int left_index = static_cast<int>(nodes.size());
        const float left_cost = build(left_prims, left_events, left_voxel, depth + 1, bad_refines);
        const int right_index = static_cast<int>(nodes.size());
        const float right_cost = build(right_prims, right_events, right_voxel, depth + 1, bad_refines);
        const auto probability = split_probability(voxel, best_axis, best_position - voxel.lo_a(best_axis),
                                                   voxel.hi_a(best_axis) - best_position);
        const float final_cost = kTraversalCost + probability.first * left_cost + probability.second * right_cost;
        if(final_cost < leaf_cost) {
            nodes[index].leaf = false;
            nodes[index].axis = best_axis;
            nodes[index].split = best_position;
            nodes[index].left = left_index;
            nodes[index].right = right_index;
            return final_cost;
        }
        make_leaf(index, prims);  // retract
        return leaf_cost;
    }

    const float* bmin_;
    const float* bmax_;
    std::vector<uint8_t> side_;
    int max_depth_ = 1;
};

uint32_t pack_node(const KdBuilder& b, int raw, PackedTree& out, uint32_t depth) {
    const uint32_t index = static_cast<uint32_t>(out.nodes.size());
    out.nodes.push_back(uint2{0u, 0u});
    out.depth = std::max(out.depth, depth);
    const RawNode& n = b.nodes[raw];
    if(n.leaf) {
        const uint32_t first = static_cast<uint32_t>(out.refs.size());
        for(int i = 0; i < n.count; ++i) out.refs.push_back(b.ordered[n.first + i]);
        out.nodes[index] = uint2{first, (static_cast<uint32_t>(n.count) << 2) | kLeafTag};
        return index;
    }
    pack_node(b, n.left, out, depth + 1);  // lands at index + 1
    const uint32_t right = pack_node(b, n.right, out, depth + 1);
    uint32_t split_bits;
    memcpy(&split_bits, &n.split, 4);
    out.nodes[index] = uint2{split_bits, (right << 2) | static_cast<uint32_t>(n.axis)};
    return index;
}

// ------------------------------------------------------------------------------------------------
// Catmull-Rom splines on uniform knots (src/material/func/catmull_rom.h, Mitsuba spline.cpp)

float interp_1d(float x, const float* values, size_t size, float mn, float mx) {
    if(!(x >= mn && x <= mx)) return 0.0f;
    float t = ((x - mn) * static_cast<float>(size - 1)) / (mx - mn);
    size_t k = static_cast<size_t>(t);
    if(k > size - 2) k = size - 2;
    const float f0 = values[k];
    const float f1 = values[k + 1];
    const float d0 = k > 0 ? 0.5f * (values[k + 1] - values[k - 1]) : (values[k + 1] - values[k]);
    const float d1 = (k + 2 < size) ? 0.5f * (values[k + 2] - values[k]) : (values[k + 1] - values[k]);
    t -= static_cast<float>(k);
    const float t2 = t * t;
    const float t3 = t2 * t;
    return (2.0f * t3 - 3.0f * t2 + 1.0f) * f0 + (-2.0f * t3 + 3.0f * t2) * f1 + (t3 - 2.0f * t2 + t) * d0 +
           (t3 - t2) * d1;
}

// knot index and the four weights of one dimension; false when p is outside [mn, mx]
bool knot_weights(float p, size_t size, float mn, float mx, size_t& knot, float w[4]) {
    if(!(p >= mn && p <= mx)) return false;
    float t = ((p - mn) * static_cast<float>(size - 1)) / (mx - mn);
    knot = std::min(static_cast<size_t>(t), size - 2);
    t -= static_cast<float>(knot);
    const float t2 = t * t;
    const float t3 = t2 * t;
    w[0] = 0.0f;
    w[1] = 2.0f * t3 - 3.0f * t2 + 1.0f;
    w[2] = -2.0f * t3 + 3.0f * t2;
    w[3] = 0.0f;
    const float d0 = t3 - 2.0f * t2 + t;
    const float d1 = t3 - t2;
    if(knot > 0) {
        w[2] += 0.5f * d0;
        w[0] -= 0.5f * d0;
    } else {
        w[2] += d0;
        w[1] -= d0;
    }
    if(knot + 2 < size) {
        w[3] += 0.5f * d1;
        w[1] -= 0.5f * d1;
    } else {
        w[2] += d1;
        w[1] -= d1;
    }
    return true;
}

float interp_2d(const float p[2], const float* values, const size_t size[2]) {
    float w[2][4];
    size_t knot[2];
    for(int d = 0; d < 2; ++d) {
        if(!knot_weights(p[d], size[d], 0.0f, 1.0f, knot[d], w[d])) return 0.0f;
    }
    float result = 0.0f;
    for(int y = -1; y <= 2; ++y) {
        const float wy = w[1][y + 1];
        for(int x = -1; x <= 2; ++x) {
            const float wxy = w[0][x + 1] * wy;
            if(wxy == 0.0f) continue;
            const size_t pos = (knot[1] + static_cast<size_t>(y)) * size[0] + knot[0] + static_cast<size_t>(x);
            result += values[pos] * wxy;
        }
    }
    return result;
}

float interp_3d(const float p[3], const float* values, const size_t size[3]) {
    float w[3][4];
    size_t knot[3];
    for(int d = 0; d < 3; ++d) {
        if(!knot_weights(p[d], size[d], 0.0f, 1.0f, knot[d], w[d])) return 0.0f;
    }
    float result = 0.0f;
    for(int z = -1; z <= 2; ++z) {
        const float wz = w[2][z + 1];
        for(int y = -1; y <= 2; ++y) {
            const float wyz = w[1][y + 1] * wz;
            for(int x = -1; x <= 2; ++x) {
                const float wxyz = w[0][x + 1] * wyz;
                if(wxyz == 0.0f) continue;
                const size_t pos = ((knot[2] + static_cast<size_t>(z)) * size[1] + (knot[1] + static_cast<size_t>(y))) *
                                       size[0] +
                                   knot[0] + static_cast<size_t>(x);
                result += values[pos] * wxyz;
            }
        }
    }
    return result;
}

bool read_u64(std::ifstream& in, uint64_t& v) {
    unsigned char b[8];
    in.read(reinterpret_cast<char*>(b), 8);
    v = 0;
    for(int i = 7; i >= 0; --i) v = (v << 8) | b[i];
    return static_cast<bool>(in);
}
bool read_f32(std::ifstream& in, float& v) {
    unsigned char b[4];
    in.read(reinterpret_cast<char*>(b), 4);
    const uint32_t bits = static_cast<uint32_t>(b[0]) | (static_cast<uint32_t>(b[1]) << 8) |
                          (static_cast<uint32_t>(b[2]) << 16) | (static_cast<uint32_t>(b[3]) << 24);
    memcpy(&v, &bits, 4);
    return static_cast<bool>(in);
}

// ------------------------------------------------------------------------------------------------
// Adaptive Gauss-Lobatto quadrature (Gander & Gautschi 2000, "Adaptive quadrature - revisited"), in
// the float form the reference uses for Fdr (src/material/func/gauss_lobatto.h, max 1024 evaluations,
// absolute error 0, relative error 1e-5).

struct Lobatto {
    size_t max_evals = 1024;
    float abs_error = 0.0f;
    float rel_error = 1e-5f;
    const float alpha = static_cast<float>(sqrt(2.0 / 3.0));
    const float beta = static_cast<float>(1.0 / sqrt(5.0));
    const float x1 = static_cast<float>(0.94288241569547971906);
    const float x2 = static_cast<float>(0.64185334234578130578);
    const float x3 = static_cast<float>(0.23638319966214988028);

    template <typename F>
    float tolerance(const F& f, float a, float b, size_t& evals) const {
        const float m = (a + b) * 0.5f;
        const float h = (b - a) * 0.5f;
        const float y1 = f(a), y3 = f(m - alpha * h), y5 = f(m - beta * h), y7 = f(m), y9 = f(m + beta * h);
        const float y11 = f(m + alpha * h), y13 = f(b);
        const float f1a = f(m - x1 * h), f1b = f(m + x1 * h);
        const float f2a = f(m - x2 * h), f2b = f(m + x2 * h);
        const float f3a = f(m - x3 * h), f3b = f(m + x3 * h);
        const float acc = h * (static_cast<float>(0.0158271919734801831) * (y1 + y13) +
                               static_cast<float>(0.0942738402188500455) * (f1a + f1b) +
                               static_cast<float>(0.1550719873365853963) * (y3 + y11) +
                               static_cast<float>(0.1888215739601824544) * (f2a + f2b) +
                               static_cast<float>(0.1997734052268585268) * (y5 + y9) +
                               static_cast<float>(0.2249264653333395270) * (f3a + f3b) +
                               static_cast<float>(0.2426110719014077338) * y7);
        evals += 13;
        float r = 1.0f;
        const float integral2 = (h / 6.0f) * (y1 + y13 + 5.0f * (y5 + y9));
        const float integral1 = (h / 1470.0f) * (77.0f * (y1 + y13) + 432.0f * (y3 + y11) + 625.0f * (y5 + y9) + 672.0f * y7);
        if(fabsf(integral2 - acc) != 0.0f) r = fabsf(integral1 - acc) / fabsf(integral2 - acc);
        if(r == 0.0f || r > 1.0f) r = 1.0f;
        const float eps = std::numeric_limits<float>::epsilon();
        float result = std::numeric_limits<float>::infinity();
        if(rel_error != 0.0f && acc != 0.0f) result = acc * smax(rel_error, eps) / (r * eps);
        if(abs_error != 0.0f) result = smin(result, abs_error / (r * eps));
        return result;
    }

    template <typename F>
    float step(const F& f, float a, float b, float fa, float fb, float acc, size_t& evals) const {
        const float h = (b - a) * 0.5f;
        const float m = (a + b) * 0.5f;
        const float mll = m - alpha * h, ml = m - beta * h, mr = m + beta * h, mrr = m + alpha * h;
        const float fmll = f(mll), fml = f(ml), fm = f(m), fmr = f(mr), fmrr = f(mrr);
        const float integral2 = (h / 6.0f) * (fa + fb + 5.0f * (fml + fmr));
        const float integral1 =
            (h / 1470.0f) * (77.0f * (fa + fb) + 432.0f * (fmll + fmrr) + 625.0f * (fml + fmr) + 672.0f * fm);
        evals += 5;
        if(evals >= max_evals) return integral1;
        const float dist = acc + (integral1 - integral2);
        if(dist == acc || mll <= a || b <= mrr) return integral1;
        const float s0 = step(f, a, mll, fa, fmll, acc, evals);
        const float s1 = step(f, mll, ml, fmll, fml, acc, evals);
        const float s2 = step(f, ml, m, fml, fm, acc, evals);
        const float s3 = step(f, m, mr, fm, fmr, acc, evals);
        const float s4 = step(f, mr, mrr, fmr, fmrr, acc, evals);
        const float s5 = step(f, mrr, b, fmrr, fb, acc, evals);
        return s0 + s1 + s2 + s3 + s4 + s5;
    }

    template <typename F>
    float integrate(const F& f, float a, float b) const {
        float factor = 1.0f;
        size_t evals = 0;
        if(a == b) return 0.0f;
        if(b < a) {
            std::swap(a, b);
            factor = -1.0f;
        }
        const float tol = tolerance(f, a, b, evals);
        evals += 2;
        return factor * step(f, a, b, f(a), f(b), tol, evals);
    }
};

float fresnel_ext_host(float cos_theta_i, float eta) {
    if(eta == 1.0f) return 0.0f;
    const float scale = cos_theta_i > 0.0f ? (1.0f / eta) : eta;
    const float cos_theta_t_sqr = 1.0f - (1.0f - cos_theta_i * cos_theta_i) * (scale * scale);
    if(cos_theta_t_sqr <= 0.0f) return 1.0f;
    const float cos_i = fabsf(cos_theta_i);
    const float cos_t = sqrtf(cos_theta_t_sqr);
    const float rs = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    const float rp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (rs * rs + rp * rp);
}

float luminance(const float* c) { return 0.212671f * c[0] + 0.715160f * c[1] + 0.072169f * c[2]; }

uint32_t bsdf_flags(const lrt_material_desc& m, const lrt_material_desc* all) {
    switch(m.type) {
    case LRT_DIFFUSE: return LRT_BSDF_DIFFUSE | LRT_BSDF_REFLECTIVE;
    case LRT_ROUGH_CONDUCTOR:
        return m.alpha <= 0.0f ? (LRT_BSDF_SPECULAR | LRT_BSDF_REFLECTIVE | LRT_BSDF_METALLIC)
                               : (LRT_BSDF_GLOSSY | LRT_BSDF_REFLECTIVE | LRT_BSDF_METALLIC);
    case LRT_DIELECTRIC:
        return LRT_BSDF_SPECULAR | LRT_BSDF_REFLECTIVE | LRT_BSDF_DIELECTRIC | LRT_BSDF_REFRACTIVE;
    case LRT_ROUGH_DIELECTRIC: return LRT_BSDF_GLOSSY | LRT_BSDF_REFLECTIVE | LRT_BSDF_REFRACTIVE | LRT_BSDF_DIELECTRIC;
    case LRT_PLASTIC: return LRT_BSDF_SPECULAR | LRT_BSDF_REFLECTIVE | LRT_BSDF_DIELECTRIC | LRT_BSDF_DIFFUSE;
    case LRT_ROUGH_PLASTIC: return LRT_BSDF_GLOSSY | LRT_BSDF_REFLECTIVE | LRT_BSDF_DIELECTRIC | LRT_BSDF_DIFFUSE;
    case LRT_COATING: return bsdf_flags(all[m.nested], all) | LRT_BSDF_SPECULAR | LRT_BSDF_REFLECTIVE | LRT_BSDF_DIELECTRIC;
    case LRT_ROUGH_COATING: return bsdf_flags(all[m.nested], all) | LRT_BSDF_GLOSSY | LRT_BSDF_REFLECTIVE | LRT_BSDF_DIELECTRIC;
    default: return 0u;
    }
}

int component_count(const lrt_material_desc& m, const lrt_material_desc* all) {
    switch(m.type) {
    case LRT_DIELECTRIC:
    case LRT_PLASTIC:
    case LRT_ROUGH_PLASTIC: return 2;
    case LRT_COATING:
    case LRT_ROUGH_COATING: return component_count(all[m.nested], all) + 1;
    default: return 1;  // bsdf::component_count default (bsdf.h:60), rough dielectric included
    }
}

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace

// ------------------------------------------------------------------------------------------------

namespace {

// Median-split hierarchy over object boxes: leaves of at most 4 objects, children ordered as built.
// The traversal visits every object whose box it may reach and resolves ties by object index, so the
// closest hit does not depend on this tree's shape.
struct TlasBuilder {
    const std::vector<Box>& boxes;
    std::vector<int32_t> idx;
    std::vector<float4>& nodes;
    std::vector<int32_t>& objs;

    static float bits(int32_t v) {
        float f;
        memcpy(&f, &v, 4);
        return f;
    }

    int32_t build(int32_t lo, int32_t hi, int depth) {
        const int32_t node = static_cast<int32_t>(nodes.size() / 2);
        nodes.push_back(float4{});
        nodes.push_back(float4{});
        Box bounds, centroids;
        for(int32_t i = lo; i < hi; ++i) {
            bounds.extend(boxes[idx[i]]);
            centroids.extend((boxes[idx[i]].lo + boxes[idx[i]].hi) * 0.5f);
        }
        const int32_t count = hi - lo;
        if(count <= 4 || depth >= kTlasStack - 2) {
            const int32_t first = static_cast<int32_t>(objs.size());
            objs.insert(objs.end(), idx.begin() + lo, idx.begin() + hi);
            nodes[2 * node] = float4{bounds.lo.x, bounds.lo.y, bounds.lo.z, bits(first)};
            nodes[2 * node + 1] = float4{bounds.hi.x, bounds.hi.y, bounds.hi.z, bits(-count)};
            return node;
        }
        const f3 ext = centroids.hi - centroids.lo;
        const int axis = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
        const int32_t mid = lo + count / 2;
        std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int32_t a, int32_t b) {
            const float ca = comp(boxes[a].lo + boxes[a].hi, axis), cb = comp(boxes[b].lo + boxes[b].hi, axis);
            return ca < cb || (ca == cb && a < b);
        });
        const int32_t left = build(lo, mid, depth + 1);
        const int32_t right = build(mid, hi, depth + 1);
        nodes[2 * node] = float4{bounds.lo.x, bounds.lo.y, bounds.lo.z, bits(left)};
        nodes[2 * node + 1] = float4{bounds.hi.x, bounds.hi.y, bounds.hi.z, bits(right)};
        return node;
    }
};

}  // namespace

KdRootInfo kd_root_info(const float* bmin, const float* bmax, uint32_t count) {
    KdRootInfo r{};
    Box root;
    uint64_t events = 0;
    for(uint32_t i = 0; i < count; ++i) {  // as KdBuilder::run
        Box b;
        b.lo = load3(bmin + 3ull * i);
        b.hi = load3(bmax + 3ull * i);
        root.extend(b);
        for(int a = 0; a < 3; ++a) events += bmin[3ull * i + a] == bmax[3ull * i + a] ? 1 : 2;
    }
    store3(r.lo, root.lo);
    store3(r.hi, root.hi);
    r.depth_limit =
        count ? std::max(std::min(48, static_cast<int>(8.0f + 1.3f * log2f(static_cast<float>(count)))), 1) : 1;
    r.n_events = events;
    return r;
}

void build_kdtree(const float* bmin, const float* bmax, uint32_t count, PackedTree& out) {
    out = PackedTree{};
    if(count == 0) {
        out.nodes.push_back(uint2{0u, (0u << 2) | kLeafTag});  // empty leaf: traversal tests nothing
        return;
    }
    KdBuilder b(bmin, bmax, count);
    b.run(count);
    pack_node(b, 0, out, 1);
}

int rough_transmittance_eta(const char* path, float eta, std::vector<float>& sliced_t, std::vector<float>& sliced_d,
                            float& alpha_min_out, float& alpha_max_out, std::string& err) {
    std::ifstream in(path, std::ios::binary);
    if(!in) {
        err = std::string("rough transmittance: missing ") + path;
        return LRT_ERR_IO;
    }
    char header[17];
    in.read(header, 17);
    if(!in || memcmp(header, "MTS_TRANSMITTANCE", 17) != 0) {
        err = std::string("rough transmittance: invalid header in ") + path;
        return LRT_ERR_IO;
    }
    uint64_t n_eta, n_alpha, n_theta;
    float eta_min, eta_max, alpha_min, alpha_max;
    if(!read_u64(in, n_eta) || !read_u64(in, n_alpha) || !read_u64(in, n_theta) || !read_f32(in, eta_min) ||
       !read_f32(in, eta_max) || !read_f32(in, alpha_min) || !read_f32(in, alpha_max)) {
        err = "rough transmittance: truncated header";
        return LRT_ERR_IO;
    }
    if(n_theta != LRT_TRANS_SAMPLES || n_eta < 2 || n_alpha < 2 || n_eta > 4096 || n_alpha > 4096) {
        err = "rough transmittance: unexpected table dimensions";
        return LRT_ERR_IO;
    }
    const size_t trans_size = 2 * n_eta * n_alpha * n_theta;
    const size_t diff_size = 2 * n_eta * n_alpha;
    std::vector<float> trans(trans_size), diff(diff_size);
    size_t dt = 0, dd = 0;
    for(size_t i = 0; i < 2 * n_eta; ++i) {
        for(size_t j = 0; j < n_alpha; ++j) {
            for(size_t k = 0; k < n_theta; ++k) {
                if(!read_f32(in, trans[dt++])) {
                    err = "rough transmittance: truncated table";
                    return LRT_ERR_IO;
                }
            }
            if(!read_f32(in, diff[dd++])) {
                err = "rough transmittance: truncated table";
                return LRT_ERR_IO;
            }
        }
    }
    // range checks (rough_transmittance.h:114-127)
    float check = eta < 1.0f ? 1.0f / eta : eta;
    if(check < eta_min || check > eta_max) {
        err = "rough transmittance: eta outside table range";
        return LRT_ERR_RANGE;
    }
    // set_eta (rough_transmittance.h:129-167)
    const float* trans_src = trans.data();
    const float* diff_src = diff.data();
    if(eta < 1.0f) {
        trans_src += n_eta * n_alpha * n_theta;
        diff_src += n_eta * n_alpha;
        eta = 1.0f / eta;
    }
    if(eta < eta_min) eta = eta_min;
    const float warped_eta = powf((eta - eta_min) / (eta_max - eta_min), 0.25f);
    const float d_alpha = 1.0f / static_cast<float>(n_alpha - 1);
    const float d_theta = 1.0f / static_cast<float>(n_theta - 1);
    const size_t size3[3] = {n_theta, n_alpha, n_eta};
    const size_t size2e[2] = {n_alpha, n_eta};
    sliced_t.assign(n_alpha * n_theta, 0.0f);
    sliced_d.assign(n_alpha, 0.0f);
    for(size_t i = 0; i < n_alpha; ++i) {
        for(size_t j = 0; j < n_theta; ++j) {
            const float p[3] = {static_cast<float>(j) * d_theta, static_cast<float>(i) * d_alpha, warped_eta};
            sliced_t[i * n_theta + j] = interp_3d(p, trans_src, size3);
        }
        const float q[2] = {static_cast<float>(i) * d_alpha, warped_eta};
        sliced_d[i] = interp_2d(q, diff_src, size2e);
    }
    alpha_min_out = alpha_min;
    alpha_max_out = alpha_max;
    return LRT_OK;
}

int rough_transmittance_alpha(const float* sliced_t, const float* sliced_d, uint32_t n_alpha, float alpha_min,
                              float alpha_max, float alpha, float* table, float* diffuse, std::string& err) {
    const size_t n_theta = LRT_TRANS_SAMPLES;
    if(n_alpha < 2 || n_alpha > 4096) {
        err = "rough transmittance: unexpected table dimensions";
        return LRT_ERR_INVALID_ARGUMENT;
    }
    if(alpha < alpha_min || alpha > alpha_max) {
        err = "rough transmittance: alpha outside table range";
        return LRT_ERR_RANGE;
    }
    const float d_theta = 1.0f / static_cast<float>(n_theta - 1);
    // set_alpha (rough_transmittance.h:169-185)
    const float warped_alpha = powf((alpha - alpha_min) / (alpha_max - alpha_min), 0.25f);
    const size_t size2a[2] = {n_theta, n_alpha};
    for(size_t i = 0; i < n_theta; ++i) {
        const float p[2] = {static_cast<float>(i) * d_theta, warped_alpha};
        table[i] = interp_2d(p, sliced_t, size2a);
    }
    const float d = interp_1d(warped_alpha, sliced_d, n_alpha, 0.0f, 1.0f);
    *diffuse = sclamp(d, 0.0f, 1.0f);  // eval_diffuse()
    return LRT_OK;
}

int rough_transmittance_slice(const char* path, float eta, float alpha, float* table, float* diffuse, std::string& err) {
    std::vector<float> sliced_t, sliced_d;
    float alpha_min = 0.0f, alpha_max = 0.0f;
    const int st = rough_transmittance_eta(path, eta, sliced_t, sliced_d, alpha_min, alpha_max, err);
    if(st != LRT_OK) return st;
    return rough_transmittance_alpha(sliced_t.data(), sliced_d.data(), static_cast<uint32_t>(sliced_d.size()), alpha_min,
                                     alpha_max, alpha, table, diffuse, err);
}

float fresnel_diffuse_reflectance(float eta) {
    const Lobatto q;
    return q.integrate([eta](float xi) { return fresnel_ext_host(sqrtf(xi), eta); }, 0.0f, 1.0f);
}

// ---- Hosek-Wilkie RGB sky state ----
#include "lrt_hosek_rgb.inc"

namespace {

// The model's quintic Bernstein blend over its six elevation control points c[0], c[step], ..., c[5 step]
// at the warped elevation s, B_k(s) = C(5,k) (1-s)^(5-k) s^k, each term multiplied and the terms summed
// in the order ArHosekSkyModel_CookConfiguration writes them (ArHosekSkyModel.cc:164-171) so that the
// double result is the reference's bit for bit.
double hosek_bernstein(const double* c, int step, double s) {
    const double r = 1.0 - s;
    return pow(r, 5.0) * c[0] + 5.0 * pow(r, 4.0) * s * c[step] + 10.0 * pow(r, 3.0) * pow(s, 2.0) * c[2 * step] +
           10.0 * pow(r, 2.0) * pow(s, 3.0) * c[3 * step] + 5.0 * r * pow(s, 4.0) * c[4 * step] +
           pow(s, 5.0) * c[5 * step];
}

// One channel: bilinear in (ground albedo 0/1, integer turbidity t/t+1) over the tables of `per` values
// per (albedo, turbidity) cell, each cell the Bernstein blend over elevation; `count` outputs.
void hosek_cook(const double* table, int per, int count, double turbidity, double albedo, double elevation,
                double* out) {
    const int t = static_cast<int>(turbidity);
    const double t_rem = turbidity - static_cast<double>(t);
    const double s = pow(elevation / (3.141592653589793 / 2.0), 1.0 / 3.0);
    const int stride = 6 * per;  // one (albedo, turbidity) cell: 6 control points x `per` values
    // cells in the reference's accumulation order: (albedo 0, t), (albedo 1, t), then -- below
    // turbidity 10 -- (albedo 0, t + 1), (albedo 1, t + 1)
    struct Cell {
        int albedo_side, turbidity;
        double weight;
    };
    const Cell cells[4] = {{0, t, (1.0 - albedo) * (1.0 - t_rem)},
                           {1, t, albedo * (1.0 - t_rem)},
                           {0, t + 1, (1.0 - albedo) * t_rem},
                           {1, t + 1, albedo * t_rem}};
    const int n_cells = t == 10 ? 2 : 4;
    for(int k = 0; k < n_cells; ++k) {
        const double* cell = table + cells[k].albedo_side * 10 * stride + (cells[k].turbidity - 1) * stride;
        for(int i = 0; i < count; ++i) {
            const double v = cells[k].weight * hosek_bernstein(cell + i, per, s);
            out[i] = k == 0 ? v : out[i] + v;
        }
    }
}

}  // namespace

int hosek_state(const float sun_direction[3], float turbidity, float albedo, double config[3][9], double radiance[3],
                std::string& error) {
    if(!(turbidity >= 1.0f && turbidity <= 10.0f)) {
        error = "turbidity must lie in [1, 10] (the model's table range)";
        return LRT_ERR_RANGE;
    }
    if(!(albedo >= 0.0f && albedo <= 1.0f)) {
        error = "ground albedo must lie in [0, 1]";
        return LRT_ERR_RANGE;
    }
    const f3 d = load3(sun_direction);
    if(!(length_squared(d) > 0.0f)) {
        error = "sun direction must be non-zero";
        return LRT_ERR_INVALID_ARGUMENT;
    }
    // env_emitter.h:14,28: the direction normalised in float, elevation = asin(clamp(y, -1, 1)) in float
    const f3 sun = normalize(d);
    const float elevation = asinf(sclamp(sun.y, -1.0f, 1.0f));
    for(int c = 0; c < 3; ++c) {
        hosek_cook(kHosekRgb[c], 9, 9, turbidity, albedo, elevation, config[c]);
        hosek_cook(kHosekRgbRad[c], 1, 1, turbidity, albedo, elevation, &radiance[c]);
    }
    return LRT_OK;
}

// Sobol direction numbers: dimension 0 is the van der Corput sequence, dimensions 1..15 come from
// the primitive polynomials and initial direction numbers of Joe & Kuo (new-joe-kuo-6.21201,
// dimensions 2..16), the table src/core/sobol.h:51-69 also uses.
void sobol_direction_table(uint32_t table[16][32]) {
    struct Poly {
        uint32_t degree, a, m[6];
    };
    static const Poly polys[15] = {
        {1, 0, {1, 0, 0, 0, 0, 0}},     {2, 1, {1, 3, 0, 0, 0, 0}},     {3, 1, {1, 3, 1, 0, 0, 0}},
        {3, 2, {1, 1, 1, 0, 0, 0}},     {4, 1, {1, 1, 3, 3, 0, 0}},     {4, 4, {1, 3, 5, 13, 0, 0}},
        {5, 2, {1, 1, 5, 5, 17, 0}},    {5, 4, {1, 1, 5, 5, 5, 0}},     {5, 7, {1, 1, 7, 11, 19, 0}},
        {5, 11, {1, 1, 5, 1, 1, 0}},    {5, 13, {1, 1, 1, 3, 11, 0}},   {5, 14, {1, 3, 5, 5, 13, 0}},
        {6, 1, {1, 3, 3, 9, 7, 49}},    {6, 13, {1, 1, 1, 15, 21, 21}}, {6, 16, {1, 3, 1, 13, 27, 49}},
    };
    for(int bit = 0; bit < 32; ++bit) table[0][bit] = 1u << (31 - bit);
    for(int d = 0; d < 15; ++d) {
        const Poly& p = polys[d];
        uint32_t m[33] = {0};
        for(uint32_t i = 1; i <= p.degree; ++i) m[i] = p.m[i - 1];
        // m_i = 2 a_1 m_{i-1} ^ 4 a_2 m_{i-2} ^ ... ^ 2^s m_{i-s} ^ m_{i-s}
        for(uint32_t i = p.degree + 1; i <= 32; ++i) {
            uint32_t v = (m[i - p.degree] << p.degree) ^ m[i - p.degree];
            for(uint32_t k = 1; k < p.degree; ++k) {
                if((p.a >> (p.degree - 1 - k)) & 1u) v ^= m[i - k] << k;
            }
            if(i < 32) v &= (1u << i) - 1u;
            m[i] = v;
        }
        for(int i = 1; i <= 32; ++i) table[d + 1][i - 1] = m[i] << (32 - i);
    }
}

// ------------------------------------------------------------------------------------------------

// ------------------------------------------------------------------------------------------------
// Wavefront OBJ, read as load_obj does (src/io/obj_loader.h:11-141): each line without its '\r';
// blank and '#' lines skipped; 'v' and 'vn' read three floats with the stream extractor; an 'f'
// corner is "p", "p/t", "p//n" or "p/t/n" with 1-based or negative (from the end) indices; a face is
// fanned from its first corner, a triangle whose cross product has zero length is dropped, and a
// corner without a normal takes the triangle's unit geometric normal. Afterwards every position is
// moved so that the box of the referenced positions is centred at the origin and scaled so that its
// longest side is 1. A missing file, an index out of range, a face of fewer than three corners or no
// triangle at all is an error.

namespace {

int obj_index(int index, int count) { return index < 0 ? count + index : index - 1; }

}  // namespace

int load_obj(const char* path, std::vector<float>& positions_out, std::vector<uint32_t>& indices,
             std::vector<float>& normals_out, std::string& err) {
    positions_out.clear();
    indices.clear();
    normals_out.clear();
    std::ifstream file(path);
    if(!file) {
        err = std::string("obj: cannot open ") + path;
        return LRT_ERR_IO;
    }
    std::vector<f3> positions, normals, corner_normals;
    std::string line;
    uint64_t line_no = 0;
    while(std::getline(file, line)) {
        ++line_no;
        if(!line.empty() && line.back() == '\r') line.pop_back();
        if(line.empty() || line[0] == '#') continue;
        std::istringstream stream(line);
        std::string tag;
        stream >> tag;
        if(tag == "v" || tag == "vn") {
            float x = 0.0f, y = 0.0f, z = 0.0f;
            stream >> x >> y >> z;
            (tag == "v" ? positions : normals).push_back(f3{x, y, z});
        } else if(tag == "f") {
            std::vector<uint32_t> face_p;
            std::vector<int> face_n;
            std::string corner;
            while(stream >> corner) {
                int pi = 0, ni = 0;
                try {
                    const size_t slash = corner.find('/');
                    if(slash == std::string::npos) {
                        pi = std::stoi(corner);
                    } else {
                        pi = std::stoi(corner.substr(0, slash));
                        const size_t slash2 = corner.find('/', slash + 1);
                        if(slash2 != std::string::npos && slash2 + 1 < corner.size()) ni = std::stoi(corner.substr(slash2 + 1));
                    }
                } catch(const std::exception&) {
                    err = "obj: line " + std::to_string(line_no) + ": malformed face corner";
                    return LRT_ERR_INVALID_ARGUMENT;
                }
                const int p = obj_index(pi, static_cast<int>(positions.size()));
                if(p < 0 || p >= static_cast<int>(positions.size())) {
                    err = "obj: line " + std::to_string(line_no) + ": position index out of range";
                    return LRT_ERR_INVALID_ARGUMENT;
                }
                face_p.push_back(static_cast<uint32_t>(p));
                int n = -1;
                if(ni != 0) {
                    n = obj_index(ni, static_cast<int>(normals.size()));
                    if(n < 0 || n >= static_cast<int>(normals.size())) {
                        err = "obj: line " + std::to_string(line_no) + ": normal index out of range";
                        return LRT_ERR_INVALID_ARGUMENT;
                    }
                }
                face_n.push_back(n);
            }
            if(face_p.size() < 3) {
                err = "obj: line " + std::to_string(line_no) + ": face with fewer than three corners";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            for(size_t k = 1; k + 1 < face_p.size(); ++k) {
                const uint32_t tri[3] = {face_p[0], face_p[k], face_p[k + 1]};
                const int tri_n[3] = {face_n[0], face_n[k], face_n[k + 1]};
                const f3 g = cross(positions[tri[1]] - positions[tri[0]], positions[tri[2]] - positions[tri[0]]);
                if(length_squared(g) <= 0.0f) continue;
                const f3 unit = g / length(g);
                for(int c = 0; c < 3; ++c) {
                    indices.push_back(tri[c]);
                    corner_normals.push_back(tri_n[c] < 0 ? unit : normals[static_cast<size_t>(tri_n[c])]);
                }
            }
        }
    }
    if(indices.empty()) {
        err = std::string("obj: no triangle in ") + path;
        return LRT_ERR_INVALID_ARGUMENT;
    }
    // centre and unitise over the referenced positions (obj_loader.h:15-38)
    f3 lo = positions[indices[0]], hi = lo;
    for(const uint32_t i : indices) {
        const f3 q = positions[i];
        lo = f3{smin(lo.x, q.x), smin(lo.y, q.y), smin(lo.z, q.z)};
        hi = f3{smax(hi.x, q.x), smax(hi.y, q.y), smax(hi.z, q.z)};
    }
    const f3 center = (lo + hi) * 0.5f;
    const f3 extent = hi - lo;
    const float longest = smax(extent.x, smax(extent.y, extent.z));
    if(longest <= 0.0f) {
        err = std::string("obj: degenerate bounds in ") + path;
        return LRT_ERR_INVALID_ARGUMENT;
    }
    const float scale = 1.0f / longest;
    positions_out.reserve(3 * positions.size());
    for(const f3 q : positions) {
        const f3 m = (q - center) * scale;
        positions_out.insert(positions_out.end(), {m.x, m.y, m.z});
    }
    normals_out.reserve(3 * corner_normals.size());
    for(const f3 n : corner_normals) normals_out.insert(normals_out.end(), {n.x, n.y, n.z});
    return LRT_OK;
}

CamRec camera_from_desc(const lrt_camera_desc& c) {
    const f3 origin = load3(c.origin);
    const f3 look_at = load3(c.look_at);
    const float radians = c.fov_degrees * kPi / 180.0f;
    const float h = tanf(radians / 2.0f);
    const float viewport_height = 2.0f * h;
    const float viewport_width = c.aspect_ratio * viewport_height;
    const float focus_dist = 1.0f;
    const f3 w = normalize(origin - look_at);
    const f3 u = normalize(cross(load3(c.up), w));
    const f3 v = cross(w, u);
    const f3 horizontal = focus_dist * viewport_width * u;
    const f3 vertical = focus_dist * viewport_height * v;
    const f3 llc = origin - horizontal / 2.0f - vertical / 2.0f - focus_dist * w;
    CamRec cam{};
    store3(cam.origin, origin);
    store3(cam.llc, llc);
    store3(cam.horizontal, horizontal);
    store3(cam.vertical, vertical);
    return cam;
}

int pack_materials(const lrt_material_desc* mats, uint32_t n, std::vector<MatRec>& out, std::vector<float>& tables,
                   std::string& err) {
    out.clear();
    tables.clear();
    if(n && !mats) {
        err = "material list is null";
        return LRT_ERR_INVALID_ARGUMENT;
    }
    for(uint32_t i = 0; i < n; ++i) {
        const lrt_material_desc& m = mats[i];
        if(m.type < LRT_DIFFUSE || m.type > LRT_ROUGH_COATING) {
            err = "material " + std::to_string(i) + ": unknown type";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        if(m.type == LRT_COATING || m.type == LRT_ROUGH_COATING) {
            if(m.nested < 0 || static_cast<uint32_t>(m.nested) >= i) {
                err = "material " + std::to_string(i) + ": nested material must precede the coating";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            const int nt = mats[m.nested].type;
            if(nt == LRT_COATING || nt == LRT_ROUGH_COATING) {
                err = "material " + std::to_string(i) + ": nested coatings are not supported";
                return LRT_ERR_INVALID_ARGUMENT;
            }
        }
        MatRec r{};
        r.type = m.type;
        r.nested = (m.type == LRT_COATING || m.type == LRT_ROUGH_COATING) ? m.nested : -1;
        r.flags = bsdf_flags(m, mats);
        r.component_count = component_count(m, mats);
        r.int_ior = m.int_ior;
        r.ext_ior = m.ext_ior;
        r.alpha = m.alpha;
        r.dist_alpha = smax(smax(m.alpha, 0.0001f), 0.0001f);
        r.thickness = m.thickness;
        r.nonlinear = m.nonlinear;
        r.table = -1;
        r.specular_component = -1;
        store3(r.diffuse, load3(m.diffuse_reflectance));
        store3(r.spec_refl, load3(m.specular_reflectance));
        store3(r.spec_trans, load3(m.specular_transmittance));
        store3(r.cond_eta, load3(m.eta));
        store3(r.cond_k, load3(m.k));
        store3(r.sigma_a, load3(m.sigma_a));
        r.sigma_zero = is_zero(load3(m.sigma_a)) ? 1 : 0;
        if(m.type == LRT_PLASTIC || m.type == LRT_ROUGH_PLASTIC) {
            if(!(m.ext_ior > 0.0f) || !(m.int_ior > 0.0f)) {
                err = "material " + std::to_string(i) + ": indices of refraction must be positive";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            r.eta = m.int_ior / m.ext_ior;
            r.inv_eta = 1.0f / (r.eta * r.eta);
            r.specular_sampling_weight =
                luminance(m.specular_reflectance) / (luminance(m.diffuse_reflectance) + luminance(m.specular_reflectance));
            r.fdr = m.type == LRT_PLASTIC ? fresnel_diffuse_reflectance(1.0f / r.eta) : m.trans_internal_diffuse;
        }
        if(m.type == LRT_COATING || m.type == LRT_ROUGH_COATING) {
            r.eta = m.int_ior / m.ext_ior;
            r.inv_eta = m.ext_ior / m.int_ior;
            if(m.eta_pair[0] > 0.0f) {
                r.eta = m.eta_pair[0];
                r.inv_eta = m.eta_pair[1];
            }
            const f3 optical = load3(m.sigma_a) * (-2.0f * m.thickness);
            const float avg = (expf(optical.x) + expf(optical.y) + expf(optical.z)) / 3.0f;
            r.specular_sampling_weight = 1.0f / (avg + 1.0f);
            r.specular_component = component_count(mats[m.nested], mats);
        }
        if(m.type == LRT_ROUGH_PLASTIC || m.type == LRT_ROUGH_COATING) {
            bool any = false;
            for(int k = 0; k < LRT_TRANS_SAMPLES; ++k) any = any || m.trans_table[k] != 0.0f;
            if(!any) {
                err = "material " + std::to_string(i) + ": rough-transmittance table is empty";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            r.table = static_cast<int32_t>(tables.size() / LRT_TRANS_SAMPLES);
            tables.insert(tables.end(), m.trans_table, m.trans_table + LRT_TRANS_SAMPLES);
        }
        out.push_back(r);
    }

    return LRT_OK;
}

namespace {

// f(i) for i in [0, n) on all host cores (items taken in order from a shared counter)
template <typename F>
void parallel_for(size_t n, F f) {
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for(size_t i = next++; i < n; i = next++) f(i);
    };
    const size_t n_threads = std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for(size_t t = 1; t < n_threads; ++t) pool.emplace_back(worker);
    worker();
    for(std::thread& t : pool) t.join();
}

}  // namespace

int build_host_scene(const lrt_scene_desc* d, HostScene& s, std::string& err, const KdBatchBuilder* kd) {
    s = HostScene{};
    if(!d) {
        err = "scene description is null";
        return LRT_ERR_INVALID_ARGUMENT;
    }
    if((d->n_objects && !d->objects) || (d->n_materials && !d->materials) || (d->n_emitters && !d->emitters)) {
        err = "scene arrays are null";
        return LRT_ERR_INVALID_ARGUMENT;
    }

    // ---- materials ----
    {
        const int st = pack_materials(d->materials, d->n_materials, s.materials, s.tables, err);
        if(st != LRT_OK) return st;
    }

    // ---- objects ----
    // the meshes' kd-trees are independent: validate every mesh, then build the trees on all host cores
    std::vector<PackedTree> trees(d->n_objects);
    std::vector<uint32_t> meshes;
    {
        for(uint32_t i = 0; i < d->n_objects; ++i) {
            const lrt_object_desc& o = d->objects[i];
            if(o.kind != LRT_OBJECT_MESH) continue;
            if(o.n_indices % 3 != 0 || (o.n_indices && (!o.indices || !o.positions || !o.corner_normals))) {
                err = "object " + std::to_string(i) + ": malformed mesh";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            for(uint32_t k = 0; k < o.n_indices; ++k) {
                if(o.indices[k] >= o.n_vertices) {
                    err = "object " + std::to_string(i) + ": vertex index out of range";
                    return LRT_ERR_INVALID_ARGUMENT;
                }
            }
            meshes.push_back(i);
        }
        // triangle boxes (aabb::extend over the corners) of every mesh, meshes in parallel; then the trees,
        // on the host per mesh (in the same pass) or by `kd` for all meshes at once
        std::vector<size_t> first(meshes.size() + 1, 0);
        for(size_t m = 0; m < meshes.size(); ++m) first[m + 1] = first[m] + d->objects[meshes[m]].n_indices / 3;
        BigVec<float> all_min(kd ? 3 * first.back() : 0), all_max(kd ? 3 * first.back() : 0);
        parallel_for(meshes.size(), [&](size_t m) {
            std::vector<float> own_min, own_max;
            {
                const lrt_object_desc& o = d->objects[meshes[m]];
                const uint32_t n_tris = o.n_indices / 3;
                float* bmin = all_min.data() + 3 * first[m];
                float* bmax = all_max.data() + 3 * first[m];
                if(!kd) {
                    own_min.resize(3ull * n_tris);
                    own_max.resize(3ull * n_tris);
                    bmin = own_min.data();
                    bmax = own_max.data();
                }
                for(uint32_t t = 0; t < n_tris; ++t) {
                    Box b;
                    for(int c = 0; c < 3; ++c) b.extend(load3(o.positions + 3ull * o.indices[3 * t + c]));
                    store3(&bmin[3ull * t], b.lo);
                    store3(&bmax[3ull * t], b.hi);
                }
                if(!kd) build_kdtree(bmin, bmax, n_tris, trees[meshes[m]]);
            }
        });
        if(kd) {
            // empty meshes get the empty leaf here; the others are built together
            std::vector<uint32_t> counts;
            std::vector<size_t> built_mesh;
            for(size_t m = 0; m < meshes.size(); ++m) {
                const uint32_t n_tris = static_cast<uint32_t>(first[m + 1] - first[m]);
                if(n_tris == 0) {
                    build_kdtree(nullptr, nullptr, 0, trees[meshes[m]]);
                } else {
                    counts.push_back(n_tris);
                    built_mesh.push_back(meshes[m]);
                }
            }
            if(!counts.empty()) {
                std::vector<PackedTree> built;
                const int st = (*kd)(counts, all_min, all_max, built, err);
                if(st != LRT_OK) return st;
                for(size_t k = 0; k < built_mesh.size(); ++k) trees[built_mesh[k]] = std::move(built[k]);
            }
        }
    }
    // every mesh's nodes, triangle records (one per leaf reference), corner normals, box and area, filled
    // on all host cores at offsets fixed in object order
    std::vector<size_t> node_off(d->n_objects + 1, 0), ref_off(d->n_objects + 1, 0), normal_off(d->n_objects + 1, 0);
    for(uint32_t i = 0; i < d->n_objects; ++i) {
        const bool mesh = d->objects[i].kind == LRT_OBJECT_MESH;
        node_off[i + 1] = node_off[i] + (mesh ? trees[i].nodes.size() : 0);
        ref_off[i + 1] = ref_off[i] + (mesh ? trees[i].refs.size() : 0);
        normal_off[i + 1] = normal_off[i] + (mesh ? static_cast<size_t>(d->objects[i].n_indices / 3) * 3 : 0);
    }
    s.nodes.resize(node_off.back());
    s.tris.resize(3 * ref_off.back());
    s.ref_prim.resize(ref_off.back());
    s.normals.resize(normal_off.back());
    std::vector<Box> mesh_box(d->n_objects);
    std::vector<float> mesh_area(d->n_objects, 0.0f);
    parallel_for(meshes.size(), [&](size_t m) {
        const uint32_t i = meshes[m];
        const lrt_object_desc& o = d->objects[i];
        const PackedTree& tree = trees[i];
        std::copy(tree.nodes.begin(), tree.nodes.end(), s.nodes.begin() + node_off[i]);
        float4* tri = s.tris.data() + 3 * ref_off[i];
        uint32_t* ref = s.ref_prim.data() + ref_off[i];
        for(const uint32_t t : tree.refs) {
            const f3 p0 = load3(o.positions + 3ull * o.indices[3 * t]);
            const f3 p1 = load3(o.positions + 3ull * o.indices[3 * t + 1]);
            const f3 p2 = load3(o.positions + 3ull * o.indices[3 * t + 2]);
            const f3 e1 = p1 - p0;
            const f3 e2 = p2 - p0;
            const float degenerate = length_squared(cross(e1, e2)) <= 0.0f ? 1.0f : 0.0f;
            *tri++ = float4{p0.x, p0.y, p0.z, degenerate};
            *tri++ = float4{e1.x, e1.y, e1.z, 0.0f};
            *tri++ = float4{e2.x, e2.y, e2.z, 0.0f};
            *ref++ = t;
        }
        const uint32_t n_tris = o.n_indices / 3;
        float4* nrm = s.normals.data() + normal_off[i];
        for(uint32_t t = 0; t < n_tris; ++t) {
            for(int c = 0; c < 3; ++c) {
                const float* n = o.corner_normals + 9ull * t + 3 * c;
                *nrm++ = float4{n[0], n[1], n[2], 0.0f};
            }
        }
        Box mb;
        for(uint32_t v = 0; v < o.n_vertices; ++v) mb.extend(load3(o.positions + 3ull * v));
        mesh_box[i] = mb;
        float area = 0.0f;
        for(uint32_t t = 0; t < n_tris; ++t) {
            const f3 p0 = load3(o.positions + 3ull * o.indices[3 * t]);
            const f3 p1 = load3(o.positions + 3ull * o.indices[3 * t + 1]);
            const f3 p2 = load3(o.positions + 3ull * o.indices[3 * t + 2]);
            area += 0.5f * length(cross(p1 - p0, p2 - p0));
        }
        mesh_area[i] = area;
    });
    Box scene_box;
    for(uint32_t i = 0; i < d->n_objects; ++i) {
        const lrt_object_desc& o = d->objects[i];
        ObjRec r{};
        r.kind = o.kind;
        r.material = o.material;
        r.emitter = -1;
        if(o.material >= static_cast<int32_t>(d->n_materials) || o.material < -1) {
            err = "object " + std::to_string(i) + ": material index out of range";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        MeshTreeInfo info{0, 0, 0};
        if(o.kind == LRT_OBJECT_MESH) {
            const uint32_t n_tris = o.n_indices / 3;
            const PackedTree& tree = trees[i];
            r.node_base = static_cast<uint32_t>(node_off[i]);
            r.ref_base = static_cast<uint32_t>(ref_off[i]);
            r.tri_base = static_cast<uint32_t>(normal_off[i] / 3);
            r.n_tris = n_tris;
            r.n_nodes = static_cast<uint32_t>(tree.nodes.size());
            const Box& mb = mesh_box[i];
            store3(r.bmin, mb.lo);
            store3(r.bmax, mb.hi);
            if(o.n_vertices) scene_box.extend(mb);
            r.area = mesh_area[i];
            info = MeshTreeInfo{static_cast<uint32_t>(tree.nodes.size()), static_cast<uint32_t>(tree.refs.size()), tree.depth};
        } else if(o.kind == LRT_OBJECT_RECTANGLE) {
            if(!finite3(o.corner) || !finite3(o.edge_u) || !finite3(o.edge_v)) {
                err = "object " + std::to_string(i) + ": rectangle is not finite";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            r.material = -1;  // rectangle::hit writes bsdf_ptr = nullptr (rectangle.h:50)
            store3(r.corner, load3(o.corner));
            store3(r.edge_u, load3(o.edge_u));
            store3(r.edge_v, load3(o.edge_v));
            const f3 n = cross(load3(o.edge_u), load3(o.edge_v));
            r.area = length(n);
            store3(r.normal, r.area > 0.0f ? n / r.area : mk(0.0f));
            Box b;
            const f3 c = load3(o.corner), u = load3(o.edge_u), v = load3(o.edge_v);
            b.extend(c);
            b.extend(c + u);
            b.extend(c + v);
            b.extend(c + u + v);
            scene_box.extend(b);
        } else if(o.kind == LRT_OBJECT_SPHERE) {
            store3(r.center, load3(o.center));
            r.radius = o.radius;
            r.area = 4.0f * kPi * o.radius * o.radius;
            Box b;
            b.extend(load3(o.center) - mk(o.radius));
            b.extend(load3(o.center) + mk(o.radius));
            scene_box.extend(b);
        } else {
            err = "object " + std::to_string(i) + ": unknown kind";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        if(r.material >= 0 && (s.materials[r.material].flags & LRT_BSDF_SPECULAR) != 0) s.has_delta_bsdf = true;
        s.objects.push_back(r);
        s.mesh_info.push_back(info);
    }
    {
        const f3 half = (scene_box.hi - scene_box.lo) * 0.5f;
        s.bounding_radius = length(half);
    }
    if(s.objects.size() > kTlasMinObjects) {
        std::vector<Box> boxes(s.objects.size());
        for(size_t i = 0; i < s.objects.size(); ++i) {
            const ObjRec& r = s.objects[i];
            Box b;
            if(r.kind == LRT_OBJECT_MESH) {
                b.extend(load3(r.bmin));
                b.extend(load3(r.bmax));
            } else if(r.kind == LRT_OBJECT_RECTANGLE) {
                const f3 c = load3(r.corner), u = load3(r.edge_u), v = load3(r.edge_v);
                b.extend(c);
                b.extend(c + u);
                b.extend(c + v);
                b.extend(c + u + v);
            } else {
                b.extend(load3(r.center) - mk(r.radius));
                b.extend(load3(r.center) + mk(r.radius));
            }
            if(!(b.lo.x <= b.hi.x)) b = Box{f3{0, 0, 0}, f3{0, 0, 0}};  // an empty mesh: a point box
            boxes[i] = b;
        }
        TlasBuilder tb{boxes, {}, s.tlas, s.tlas_objs};
        tb.idx.resize(s.objects.size());
        for(size_t i = 0; i < s.objects.size(); ++i) tb.idx[i] = static_cast<int32_t>(i);
        tb.build(0, static_cast<int32_t>(s.objects.size()), 0);
    }
    {
        std::vector<std::pair<uint32_t, int32_t>> heavy;
        for(size_t i = 0; i < s.objects.size(); ++i) {
            if(s.objects[i].kind == LRT_OBJECT_MESH && s.objects[i].n_tris > 64) {
                heavy.push_back({s.objects[i].n_tris, static_cast<int32_t>(i)});
            }
        }
        if(!heavy.empty() && heavy.size() <= 4) {
            std::sort(heavy.begin(), heavy.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
            s.n_heavy = static_cast<int32_t>(heavy.size());
            for(size_t i = 0; i < heavy.size(); ++i) s.heavy[i] = heavy[i].second;
        }
    }

    // ---- emitters ----
    float sum = 0.0f;
    for(uint32_t i = 0; i < d->n_emitters; ++i) {
        const lrt_emitter_desc& e = d->emitters[i];
        EmitRec r{};
        r.kind = e.kind;
        r.object = -1;
        if(e.kind == LRT_EMITTER_AREA) {
            if(e.object < 0 || static_cast<uint32_t>(e.object) >= d->n_objects) {
                err = "emitter " + std::to_string(i) + ": object index out of range";
                return LRT_ERR_INVALID_ARGUMENT;
            }
            const ObjRec& o = s.objects[e.object];
            if(o.kind == LRT_OBJECT_MESH) {
                // triangle_mesh ctor (triangle_mesh.h:14-28): the area CDF summed triangle by triangle in
                // float, the same sum that gives the mesh's area
                const lrt_object_desc& od = d->objects[e.object];
                r.tri_first = static_cast<uint32_t>(s.light_cdf.size());
                r.n_tris = od.n_indices / 3;
                float running = 0.0f;
                for(uint32_t t = 0; t < r.n_tris; ++t) {
                    const f3 p0 = load3(od.positions + 3ull * od.indices[3 * t]);
                    const f3 p1 = load3(od.positions + 3ull * od.indices[3 * t + 1]);
                    const f3 p2 = load3(od.positions + 3ull * od.indices[3 * t + 2]);
                    running += 0.5f * length(cross(p1 - p0, p2 - p0));
                    s.light_cdf.push_back(running);
                    s.light_tri.push_back(float4{p0.x, p0.y, p0.z, 0.0f});
                    s.light_tri.push_back(float4{p1.x, p1.y, p1.z, 0.0f});
                    s.light_tri.push_back(float4{p2.x, p2.y, p2.z, 0.0f});
                }
            }
            r.object = e.object;
            r.shape = o.kind;
            r.area = o.area;
            store3(r.radiance, load3(e.radiance));
            s.objects[e.object].emitter = static_cast<int32_t>(i);  // area_emitter ctor: shape->set_emitter(this)
            // Mitsuba AreaLight power: radiance * pi * area (area_emitter.h:141-147)
            const f3 power = r.area > 0.0f ? load3(e.radiance) * (kPi * r.area) : mk(0.0f);
            const float pw[3] = {power.x, power.y, power.z};
            const float weight = luminance(pw);
            if(weight > 0.0f) {
                sum += weight;
                s.emission_index.push_back(static_cast<int32_t>(i));
                s.emission_cdf.push_back(sum);
            }
        } else if(e.kind == LRT_EMITTER_ENV) {
            const f3 sun = normalize(load3(e.sun_direction));
            store3(r.sun, sun);
            const Onb frame = onb_from_normal(sun);
            store3(r.frame[0], frame.a0);
            store3(r.frame[1], frame.a1);
            store3(r.frame[2], frame.a2);
            r.sun_active = sun.y > 0.0f ? 1 : 0;
            const double radius = 0.255 * 3.14159265358979323846 / 180.0;
            const double cosine = cos(radius);
            r.cos_cutoff = static_cast<float>(cosine);
            r.cone_pdf = static_cast<float>(1.0 / (2.0 * 3.14159265358979323846 * (1.0 - cosine)));
            r.scale = e.scale;
            bool any = false;
            for(int c = 0; c < 3; ++c) {
                for(int k = 0; k < 9; ++k) {
                    r.cfg[c][k] = e.hosek_config[c][k];
                    any = any || e.hosek_config[c][k] != 0.0;
                }
                r.rad[c] = e.hosek_radiance[c];
            }
            if(!any) {  // no state given: cook it from (sun direction, turbidity, albedo) as env_emitter does
                std::string cook_err;
                const int st = hosek_state(e.sun_direction, e.turbidity, e.albedo, r.cfg, r.rad, cook_err);
                if(st != LRT_OK) {
                    err = "emitter " + std::to_string(i) + ": " + cook_err;
                    return st;
                }
            }
            ++s.n_infinite;
        } else {
            err = "emitter " + std::to_string(i) + ": unknown kind";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        s.emitters.push_back(r);
    }
    s.emission_power = sum;

    s.cam = camera_from_desc(d->camera);
    if(s.nodes.empty()) s.nodes.push_back(uint2{0u, kLeafTag});
    if(s.tris.empty()) s.tris.push_back(float4{0, 0, 0, 1.0f});
    if(s.ref_prim.empty()) s.ref_prim.push_back(0u);
    if(s.normals.empty()) s.normals.push_back(float4{0, 0, 0, 0});
    if(s.tables.empty()) s.tables.assign(LRT_TRANS_SAMPLES, 0.0f);
    return LRT_OK;
}

}  // namespace lrt
