// Scene construction on the CPU: the balloon's latex, the shape it takes filled with water and
// hanging from its knot, its mesh, the water particles, the bullets' bodies and surfaces, and
// the initial world of a simulation.
//
// Restates src/balloon.rs (build, inflate, shoot, icosphere, spatial_order), src/bullet.rs
// (outline, surface, hull, initial), src/flight.rs (Body::new, profile), src/params.rs and
// src/presets.rs, and the setup half of Sim::new (src/sim.rs:208-441). Arithmetic keeps the
// reference's types: f64 for the inflation and the bullets, f32 where the reference uses glam's
// Vec3 (the icosphere and its ordering).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <optional>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "world.hpp"

namespace ntr {
namespace {

constexpr double PI = 3.14159265358979323846;
constexpr double TAU = 2.0 * PI;

// ---- small vector types with the reference's arithmetic order -----------------------------
struct V3f {
    float x, y, z;
};
static inline V3f operator+(V3f a, V3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3f operator-(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3f operator*(V3f a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3f operator/(V3f a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline float dot(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3f cross(V3f a, V3f b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
static inline V3f normalize(V3f a) {
    float r = 1.0f / std::sqrt(dot(a, a));
    return a * r;
}
static inline V3f normalize_or(V3f a, V3f fb) {
    float r = 1.0f / std::sqrt(dot(a, a));
    if (std::isfinite(r) && r > 0.0f) return a * r;
    return fb;
}
// Duff et al., "Building an Orthonormal Basis, Revisited" (JCGT 2017): the second vector of
// the basis around a unit `n`.
static inline V3f any_orthonormal(V3f n) {
    float sign = std::copysign(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    return {b, sign + n.y * n.y * a, -n.y};
}

struct V3d {
    double x, y, z;
};
static inline V3d operator+(V3d a, V3d b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3d operator-(V3d a, V3d b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3d operator*(V3d a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline double dot(V3d a, V3d b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3d cross(V3d a, V3d b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
static inline double length(V3d a) { return std::sqrt(dot(a, a)); }
static inline V3d normalize(V3d a) {
    double r = 1.0 / std::sqrt(dot(a, a));
    return a * r;
}
static inline V3d widen(V3f a) { return {a.x, a.y, a.z}; }

// ---- latex (src/balloon.rs:13-71) --------------------------------------------------------
constexpr double RHO_WATER = 1000.0;
constexpr double RHO_RUBBER = 950.0;
constexpr double OGDEN_MU[3] = {0.63e6, 0.0012e6, -0.01e6};
constexpr double OGDEN_AL[3] = {1.3, 5.0, -2.0};
constexpr double NECK = 0.25;

// pow(x, alpha) for the three Ogden exponents and pow(x, -0.5), for the few distinct stretches
// one evaluation of the shape's ODE asks for (its finite differences share most of them). Kept
// by the bits of x, so every value is the one pow returns.
class Powers {
   public:
    using P3 = std::array<double, 3>;
    P3 ogden(double x) {
        const uint64_t b = bits(x);
        for (int i = 0; i < n3_; i++)
            if (k3_[i] == b) return v3_[i];
        P3 v = {std::pow(x, OGDEN_AL[0]), std::pow(x, OGDEN_AL[1]), std::pow(x, OGDEN_AL[2])};
        if (n3_ < CAP) k3_[n3_] = b, v3_[n3_++] = v;
        return v;
    }
    double inv_sqrt(double x) {
        const uint64_t b = bits(x);
        for (int i = 0; i < nh_; i++)
            if (kh_[i] == b) return vh_[i];
        double v = std::pow(x, -0.5);
        if (nh_ < CAP) kh_[nh_] = b, vh_[nh_++] = v;
        return v;
    }

   private:
    static constexpr int CAP = 16;
    static uint64_t bits(double x) {
        uint64_t u;
        std::memcpy(&u, &x, 8);
        return u;
    }
    uint64_t k3_[CAP], kh_[CAP];
    P3 v3_[CAP];
    double vh_[CAP];
    int n3_ = 0, nh_ = 0;
};

struct Latex {
    double mu[3];
    double thickness;
    Latex(double shear, double thick) : thickness(thick) {
        double g0 = 0.0;
        for (int i = 0; i < 3; i++) g0 += OGDEN_MU[i] * OGDEN_AL[i];
        g0 /= 2.0;
        for (int i = 0; i < 3; i++) mu[i] = OGDEN_MU[i] * shear / g0;
    }
    // sum_i mu_i (a^alpha_i - b^alpha_i), from the powers of a and b.
    double sigma(const Powers::P3& a, const Powers::P3& b) const {
        double s = 0.0;
        for (int i = 0; i < 3; i++) s += mu[i] * (a[i] - b[i]);
        return s;
    }
    // Principal tensions (stress times deformed thickness) at stretches l1, l2; with `both`
    // false only the first is computed (the second is returned as 0 times the thickness factor).
    std::pair<double, double> tension(double l1, double l2, Powers& pw, bool both = true) const {
        double major = std::max(l1, l2), minor = std::min(l1, l2);
        double s1 = 0.0, s2 = 0.0;
        if (major > 1.0) {
            double natural = pw.inv_sqrt(major);
            if (minor < natural) {
                double s = sigma(pw.ogden(major), pw.ogden(natural));
                (l1 >= l2 ? s1 : s2) = s;
            } else {
                double l3 = 1.0 / (l1 * l2);
                const Powers::P3 p3 = pw.ogden(l3);
                s1 = sigma(pw.ogden(l1), p3);
                if (both) s2 = sigma(pw.ogden(l2), p3);
            }
        }
        double t = thickness / (l1 * l2);
        return {s1 * t, s2 * t};
    }
};

// ---- inflation (src/balloon.rs:73-248) ---------------------------------------------------
struct Sample {
    double angle, r, z;
};
struct Profile {
    std::vector<Sample> samples;
    double neck_angle = 0, z_neck = 0, neck_r = 0, volume = 0, z_centroid = 0, stretch = 0;
    double z_top() const { return z_neck; }
    double r_at(double z) const {
        const auto& s = samples;
        if (z <= 0.0 || z >= z_neck) return 0.0;
        size_t i = std::partition_point(s.begin(), s.end(), [&](const Sample& p) { return p.z < z; }) - s.begin();
        i = std::clamp<size_t>(i, 1, s.size() - 1);
        const Sample &a = s[i - 1], &b = s[i];
        return a.r + (b.r - a.r) * (z - a.z) / std::max(b.z - a.z, 1e-15);
    }
    std::pair<double, double> place(double angle) const {
        const auto& s = samples;
        size_t i = std::partition_point(s.begin(), s.end(), [&](const Sample& p) { return p.angle < angle; }) - s.begin();
        i = std::clamp<size_t>(i, 1, s.size() - 1);
        const Sample &a = s[i - 1], &b = s[i];
        double f = std::clamp((angle - a.angle) / (b.angle - a.angle), 0.0, 1.0);
        return {a.r + (b.r - a.r) * f, a.z + (b.z - a.z) * f};
    }
};

constexpr int SHOOT_STEPS = 400;
using Y5 = std::array<double, 5>;

struct ShotResult {
    std::vector<Sample> samples;
    double volume;
};

std::optional<ShotResult> shoot(const Latex& latex, double rest_r, double apex_stretch, double apex_curv, double rho_g) {
    const double neck_angle = PI - std::asin(NECK);
    Powers apex;
    const double p_apex = 2.0 * latex.tension(apex_stretch, apex_stretch, apex).first * apex_curv;
    auto deriv = [&](double th, const Y5& y) -> std::optional<Y5> {
        double r = y[0], z = y[1], psi = y[2], l1 = y[3];
        double rr = rest_r * std::sin(th);
        double l2 = r / rr;
        if (!(r > 0.0 && l1 > 0.0)) return std::nullopt;
        Powers pw;
        auto t = latex.tension(l1, l2, pw);
        double t1 = t.first, t2 = t.second;
        if (t1 <= 0.0) return std::nullopt;
        double e = 1e-6;
        double t1_l1 =
            (latex.tension(l1 * (1.0 + e), l2, pw, false).first - latex.tension(l1 * (1.0 - e), l2, pw, false).first) / (2.0 * e * l1);
        double t1_l2 =
            (latex.tension(l1, l2 * (1.0 + e), pw, false).first - latex.tension(l1, l2 * (1.0 - e), pw, false).first) / (2.0 * e * l2);
        double p = p_apex - rho_g * z;
        double dr = l1 * std::cos(psi);
        double dz = l1 * std::sin(psi);
        double dpsi = l1 * (p - t2 * std::sin(psi) / r) / t1;
        double dl2 = (dr - l2 * std::cos(th)) / rr;
        double dl1 = (dr * (t2 - t1) - r * t1_l2 * dl2) / (r * t1_l1);
        Y5 d = {dr, dz, dpsi, dl1, PI * r * r * dz};
        for (auto& v : d) v = v * rest_r;
        return d;
    };
    const double th0 = 1e-3;
    double r = apex_stretch * rest_r * std::sin(th0);
    Y5 y = {r, 0.5 * apex_curv * r * r, apex_curv * r, apex_stretch, 0.0};
    double h = (neck_angle - th0) / SHOOT_STEPS;
    double th = th0;
    ShotResult out;
    out.samples.reserve(SHOOT_STEPS + 2);
    out.samples.push_back({0.0, 0.0, 0.0});
    out.samples.push_back({th, y[0], y[1]});
    auto add = [](const Y5& a, const Y5& k, double s) {
        Y5 o;
        for (int i = 0; i < 5; i++) o[i] = a[i] + s * k[i];
        return o;
    };
    for (int it = 0; it < SHOOT_STEPS; it++) {
        auto k1 = deriv(th, y);
        if (!k1) return std::nullopt;
        auto k2 = deriv(th + 0.5 * h, add(y, *k1, 0.5 * h));
        if (!k2) return std::nullopt;
        auto k3 = deriv(th + 0.5 * h, add(y, *k2, 0.5 * h));
        if (!k3) return std::nullopt;
        auto k4 = deriv(th + h, add(y, *k3, h));
        if (!k4) return std::nullopt;
        Y5 n;
        for (int i = 0; i < 5; i++) n[i] = y[i] + h / 6.0 * ((*k1)[i] + 2.0 * (*k2)[i] + 2.0 * (*k3)[i] + (*k4)[i]);
        y = n;
        th += h;
        if (y[0] <= 0.0 || y[2] > 3.5) return std::nullopt;
        out.samples.push_back({th, y[0], y[1]});
    }
    out.volume = y[4];
    return out;
}

bool inflate_solve(const Latex& latex, double rest_r, double volume, double rho_g, Profile& prof, std::string& err);

// Inflation depends only on the latex, the rest radius, the volume and the water's weight, and
// takes about a second (hundreds of shooting integrations); the reference redoes it whenever a
// scene is rebuilt, also when only the shots or the resolution changed. Results are kept per
// exact inputs (their bits), so a rebuild of the same balloon gets the same profile at once.
bool inflate(const Latex& latex, double rest_r, double volume, double rho_g, Profile& prof, std::string& err) {
    using Key = std::array<uint64_t, 7>;
    static std::mutex mu;
    static std::map<Key, Profile> memo;
    auto bits = [](double d) {
        uint64_t u;
        std::memcpy(&u, &d, 8);
        return u;
    };
    const Key k = {bits(latex.mu[0]), bits(latex.mu[1]), bits(latex.mu[2]), bits(latex.thickness), bits(rest_r), bits(volume),
                   bits(rho_g)};
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = memo.find(k);
        if (it != memo.end()) {
            prof = it->second;
            return true;
        }
    }
    if (!inflate_solve(latex, rest_r, volume, rho_g, prof, err)) return false;
    std::lock_guard<std::mutex> g(mu);
    if (memo.size() >= 256) memo.erase(memo.begin());
    memo.emplace(k, prof);
    return true;
}

// A few threads that run a batch of independent jobs together; the calling thread takes part,
// so a pool of n runs n jobs at a time.
class Pool {
   public:
    explicit Pool(unsigned n) {
        for (unsigned i = 1; i < n; i++) th_.emplace_back([this] { work(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        wake_.notify_all();
        for (auto& t : th_) t.join();
    }
    unsigned size() const { return (unsigned)th_.size() + 1; }
    // Runs fn(i) for every i in [0, n) and returns when all have run.
    void run(size_t n, const std::function<void(size_t)>& fn) {
        if (n == 0) return;
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &fn, n_ = n, next_ = 0, left_ = n, gen_++;
        }
        wake_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return left_ == 0; });
        fn_ = nullptr;
    }

   private:
    void drain() {
        for (;;) {
            size_t i;
            const std::function<void(size_t)>* f;
            {
                std::lock_guard<std::mutex> g(mu_);
                if (!fn_ || next_ >= n_) return;
                i = next_++, f = fn_;
            }
            (*f)(i);
            std::lock_guard<std::mutex> g(mu_);
            if (--left_ == 0) done_.notify_all();
        }
    }
    void work() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                wake_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            drain();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable wake_, done_;
    const std::function<void(size_t)>* fn_ = nullptr;
    size_t n_ = 0, next_ = 0, left_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// The outcome of one shot (its end radius and volume), kept per exact inputs (apex stretch and
// log apex curvature, as bits). The search below is the reference's sequential one and reads its
// shots from here; before each of its steps the shots that step and the next are likely to need
// are run together on the pool. A shot is a pure function of its inputs, so the profile is
// bit-identical to one computed shot by shot, whatever was run ahead and on which thread.
class Shots {
   public:
    struct End {
        bool ok;
        double r, volume;
    };
    using X = std::array<double, 2>;
    Shots(const Latex& latex, double rest_r, double rho_g, unsigned threads)
        : latex_(latex), rest_r_(rest_r), rho_g_(rho_g), pool_(threads) {}
    unsigned width() const { return pool_.size(); }
    const End& get(X x) {
        auto it = memo_.find(key(x));
        if (it != memo_.end()) return it->second;
        return memo_.emplace(key(x), one(x)).first->second;
    }
    // Runs the shots not run yet, all at once (nothing on a pool of one: get() runs them then).
    void ahead(const std::vector<X>& xs) {
        if (pool_.size() < 2) return;
        std::vector<X> todo;
        for (const X& x : xs)
            if (!memo_.count(key(x)) &&
                std::none_of(todo.begin(), todo.end(), [&](const X& t) { return key(t) == key(x); }))
                todo.push_back(x);
        std::vector<End> out(todo.size());
        pool_.run(todo.size(), [&](size_t i) { out[i] = one(todo[i]); });
        for (size_t i = 0; i < todo.size(); i++) memo_.emplace(key(todo[i]), out[i]);
    }

   private:
    static std::pair<uint64_t, uint64_t> key(X x) {
        uint64_t a, b;
        std::memcpy(&a, &x[0], 8);
        std::memcpy(&b, &x[1], 8);
        return {a, b};
    }
    End one(X x) const {
        auto s = shoot(latex_, rest_r_, x[0], std::exp(x[1]), rho_g_);
        if (!s) return {false, 0.0, 0.0};
        return {true, s->samples.back().r, s->volume};
    }
    const Latex& latex_;
    double rest_r_, rho_g_;
    Pool pool_;
    std::map<std::pair<uint64_t, uint64_t>, End> memo_;
};

// Threads for the inflation's shots: NATRAY_BUILD_THREADS when set (1 runs them one by one, in
// the reference's order), else the host's, at most 8 (the search runs at most 8 ahead).
static unsigned build_threads() {
    if (const char* e = std::getenv("NATRAY_BUILD_THREADS")) {
        long n = std::strtol(e, nullptr, 10);
        if (n >= 1) return (unsigned)std::min(n, 64L);
    }
    return std::clamp(std::thread::hardware_concurrency(), 1u, 8u);
}

bool inflate_solve(const Latex& latex, double rest_r, double volume, double rho_g, Profile& prof, std::string& err) {
    const double neck_r = NECK * rest_r;
    Shots shots(latex, rest_r, rho_g, build_threads());
    const unsigned width = shots.width();
    auto miss = [&](std::array<double, 2> x, double target) -> std::optional<std::array<double, 2>> {
        const Shots::End& s = shots.get(x);
        if (!s.ok) return std::nullopt;
        return std::array<double, 2>{(s.r - neck_r) / neck_r, std::log(s.volume) - target};
    };
    const double la0 = 1.2;
    double lo = std::log(1e-3 / rest_r), hi = std::log(1e3 / rest_r);
    // 60 halvings of the apex curvature; `depth` of them at a time read shots run together, all
    // 2^depth - 1 midpoints the next `depth` halvings can reach.
    int depth = 1;
    while ((2u << depth) - 1 <= width) depth++;
    for (int i = 0; i < 60;) {
        const int k = std::min(depth, 60 - i);
        std::vector<std::pair<double, double>> tree(size_t(1) << k);
        std::vector<Shots::X> mids;
        tree[1] = {lo, hi};
        for (size_t j = 1; j < tree.size(); j++) {
            double mid = 0.5 * (tree[j].first + tree[j].second);
            mids.push_back({la0, mid});
            if (2 * j < tree.size()) tree[2 * j] = {tree[j].first, mid}, tree[2 * j + 1] = {mid, tree[j].second};
        }
        shots.ahead(mids);
        for (int m = 0; m < k; m++, i++) {
            double mid = 0.5 * (lo + hi);
            const Shots::End& s = shots.get({la0, mid});
            if (s.ok && s.r > neck_r)
                lo = mid;
            else
                hi = mid;
        }
    }
    std::array<double, 2> x = {la0, lo};
    if (!shots.get(x).ok) {
        err = "balloon doesn't inflate";
        return false;
    }
    double v = std::log(shots.get(x).volume);
    std::array<double, 2> prev = x;
    size_t n_inc = (size_t)std::max(std::ceil(std::fabs(std::log(volume) - v) / 0.05), 1.0);
    double inc = (std::log(volume) - v) / (double)n_inc;
    const double e = 1e-6;
    for (size_t step = 0; step < n_inc; step++) {
        double target = v + inc;
        std::array<double, 2> y = step > 0 ? std::array<double, 2>{2.0 * x[0] - prev[0], 2.0 * x[1] - prev[1]} : x;
        bool done = false;
        for (int it = 0; it < 30; it++) {
            shots.ahead({y, {y[0] + e, y[1]}, {y[0], y[1] + e}});
            auto f = miss(y, target);
            if (!f) break;
            double norm = std::hypot((*f)[0], (*f)[1]);
            if (norm < 1e-9) {
                done = true;
                break;
            }
            auto fa = miss({y[0] + e, y[1]}, target);
            auto fb = miss({y[0], y[1] + e}, target);
            if (!fa || !fb) break;
            double j00 = ((*fa)[0] - (*f)[0]) / e, j01 = ((*fb)[0] - (*f)[0]) / e;
            double j10 = ((*fa)[1] - (*f)[1]) / e, j11 = ((*fb)[1] - (*f)[1]) / e;
            double det = j00 * j11 - j01 * j10;
            double d0 = (-(*f)[0] * j11 + (*f)[1] * j01) / det;
            double d1 = (-(*f)[1] * j00 + (*f)[0] * j10) / det;
            // Ahead: the full Newton step with the Jacobian around it; if the full step converges,
            // the first shots of the next continuation step (extrapolated from it); shorter steps
            // of the line search with what room is left.
            const std::array<double, 2> c1 = {y[0] + 1.0 * d0, y[1] + 1.0 * d1};
            std::vector<Shots::X> next = {c1, {c1[0] + e, c1[1]}, {c1[0], c1[1] + e}};
            if (step + 1 < n_inc) {
                const Shots::X y2 = {2.0 * c1[0] - x[0], 2.0 * c1[1] - x[1]};
                next.insert(next.end(), {y2, {y2[0] + e, y2[1]}, {y2[0], y2[1] + e}});
            }
            for (double a = 0.5; a > 1e-4 && next.size() < width; a *= 0.5) next.push_back({y[0] + a * d0, y[1] + a * d1});
            shots.ahead(next);
            double a = 1.0;
            bool moved = false;
            while (a > 1e-4) {
                std::array<double, 2> c = {y[0] + a * d0, y[1] + a * d1};
                auto g = miss(c, target);
                if (g && std::hypot((*g)[0], (*g)[1]) < norm) {
                    y = c;
                    moved = true;
                    break;
                }
                a *= 0.5;
            }
            // Where the line search finds nothing, every later iteration repeats this one exactly.
            if (!moved) break;
        }
        if (!done) {
            char buf[128];
            snprintf(buf, sizeof buf, "the balloon shape didn't converge at %.3f L", std::exp(target) * 1e3);
            err = buf;
            return false;
        }
        prev = x;
        x = y;
        v = target;
    }
    auto fin = shoot(latex, rest_r, x[0], std::exp(x[1]), rho_g);
    if (!fin) {
        err = "final balloon shape failed";
        return false;
    }
    double zmom = 0.0;
    const auto& smp = fin->samples;
    for (size_t i = 0; i + 1 < smp.size(); i++) {
        const Sample &a = smp[i], &b = smp[i + 1];
        zmom += PI * 0.5 * (a.r * a.r + b.r * b.r) * (b.z - a.z) * 0.5 * (a.z + b.z);
    }
    double stretch = 0.0;
    for (size_t i = 1; i < smp.size(); i++) stretch = std::max(stretch, smp[i].r / std::max(rest_r * std::sin(smp[i].angle), 1e-12));
    prof.samples = smp;
    prof.neck_angle = smp.back().angle;
    prof.z_neck = smp.back().z;
    prof.neck_r = neck_r;
    prof.volume = fin->volume;
    prof.z_centroid = zmom / fin->volume;
    prof.stretch = stretch;
    return true;
}

// ---- mesh (src/balloon.rs:250-322) -------------------------------------------------------
struct Rng {
    uint64_t s;
    double next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) / (double)(1ull << 53);
    }
};

void icosphere(uint32_t level, std::vector<V3f>& v, std::vector<std::array<uint32_t, 3>>& f) {
    const float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    const float base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                               {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    v.clear();
    for (auto& b : base) v.push_back(normalize(V3f{b[0], b[1], b[2]}));
    f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
         {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
         {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (uint32_t l = 0; l < level; l++) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> cache;
        auto mid = [&](uint32_t a, uint32_t b) -> uint32_t {
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = cache.find(key);
            if (it != cache.end()) return it->second;
            v.push_back(normalize((v[a] + v[b]) * 0.5f));
            uint32_t idx = (uint32_t)v.size() - 1;
            cache.emplace(key, idx);
            return idx;
        };
        std::vector<std::array<uint32_t, 3>> nf;
        nf.reserve(f.size() * 4);
        for (auto& tri : f) {
            uint32_t a = tri[0], b = tri[1], c = tri[2];
            uint32_t ab = mid(a, b);
            uint32_t bc = mid(b, c);
            uint32_t ca = mid(c, a);
            nf.push_back({a, ab, ca});
            nf.push_back({b, bc, ab});
            nf.push_back({c, ca, bc});
            nf.push_back({ab, bc, ca});
        }
        f.swap(nf);
    }
}

static inline uint32_t spread10(uint32_t x) {
    x &= 0x3ff;
    x = (x | (x << 16)) & 0x030000ff;
    x = (x | (x << 8)) & 0x0300f00f;
    x = (x | (x << 4)) & 0x030c30c3;
    return (x | (x << 2)) & 0x09249249;
}
static inline uint32_t sat_u32(float f) {
    // Rust's `as u32` saturates and maps NaN to 0.
    if (!(f > 0.0f)) return 0;
    if (f >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)f;
}
static inline uint32_t morton_key(V3f p) {
    V3f q = (p * 0.5f + V3f{0.5f, 0.5f, 0.5f}) * 1023.0f;
    return spread10(sat_u32(q.x)) | spread10(sat_u32(q.y)) << 1 | spread10(sat_u32(q.z)) << 2;
}

void spatial_order(std::vector<V3f>& v, std::vector<std::array<uint32_t, 3>>& f) {
    std::vector<uint32_t> order(v.size());
    for (uint32_t i = 0; i < v.size(); i++) order[i] = i;
    std::vector<uint32_t> keys(v.size());
    for (size_t i = 0; i < v.size(); i++) keys[i] = morton_key(v[i]);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    std::vector<uint32_t> new_index(v.size());
    for (uint32_t n = 0; n < order.size(); n++) new_index[order[n]] = n;
    std::vector<V3f> nv(v.size());
    for (size_t n = 0; n < order.size(); n++) nv[n] = v[order[n]];
    v.swap(nv);
    for (auto& t : f)
        for (auto& i : t) i = new_index[i];
    std::vector<uint32_t> fk(f.size());
    for (size_t i = 0; i < f.size(); i++) fk[i] = morton_key((v[f[i][0]] + v[f[i][1]] + v[f[i][2]]) / 3.0f);
    std::vector<uint32_t> fo(f.size());
    for (uint32_t i = 0; i < f.size(); i++) fo[i] = i;
    std::stable_sort(fo.begin(), fo.end(), [&](uint32_t a, uint32_t b) { return fk[a] < fk[b]; });
    std::vector<std::array<uint32_t, 3>> nf(f.size());
    for (size_t i = 0; i < fo.size(); i++) nf[i] = f[fo[i]];
    f.swap(nf);
}

struct GpuTri {
    uint32_t v[3];
    float rest_area;
    float dm_inv[4];
};
static_assert(sizeof(GpuTri) == 32, "GpuTri is 32 bytes");

struct Balloon {
    Profile profile;
    Latex latex{1, 1};
    double bottom_y = 0;
    V3f center{};
    V3f knot{};
    double radius_max = 0;
    double spacing = 0;
    std::vector<std::array<float, 4>> particles;
    std::vector<std::array<float, 4>> mem_pos;
    std::vector<float> mem_mass;
    std::vector<GpuTri> tris;
    std::vector<uint32_t> vtri_off, vtri;

    // Where a straight line through `aim` along `dir` first meets the undisturbed balloon,
    // src/balloon.rs:466-477.
    std::optional<V3f> entry(V3f aim, V3f dir) const {
        auto inside = [&](double s) {
            V3f q = aim + dir * (float)s;
            return std::hypot((double)q.x, (double)q.z) < profile.r_at((double)q.y - bottom_y);
        };
        double reach = 1.5 * (radius_max + profile.z_top());
        const int steps = 8000;
        for (int i = 0; i <= steps; i++) {
            double s = -reach + 2.0 * reach * (double)i / (double)steps;
            if (inside(s)) return aim + dir * (float)s;
        }
        return std::nullopt;
    }
};

static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

bool build_balloon(const ntr_sim_params& p, Balloon& out, std::string& err) {
    double d = (double)p.balloon_diameter_cm * 0.01;
    double volume = PI / 6.0 * d * d * d;
    double t0 = (double)p.rubber_thickness_mm * 1e-3;
    Latex latex((double)p.rubber_modulus_mpa * 1e6, t0);
    double rest_r = (double)p.rubber_rest_diameter_cm * 0.005;
    Profile profile;
    if (!inflate(latex, rest_r, volume, RHO_WATER * (double)std::max(p.gravity, 0.0f), profile, err)) return false;
    double bottom_y = (double)p.balloon_height - profile.z_centroid;
    double radius_max = 0.0;
    for (auto& q : profile.samples) radius_max = std::max(radius_max, q.r);
    V3f center{0.0f, p.balloon_height, 0.0f};
    V3f knot{0.0f, (float)(bottom_y + profile.z_neck + 0.5 * profile.neck_r), 0.0f};

    std::vector<V3f> sphere;
    std::vector<std::array<uint32_t, 3>> faces;
    icosphere(p.mesh_level, sphere, faces);
    spatial_order(sphere, faces);
    Rng rng{p.seed == 0 ? 0x9E3779B97F4A7C15ull : splitmix64(p.seed)};
    if (rng.s == 0) rng.s = 0x9E3779B97F4A7C15ull;
    const float edge_angle = 1.1f / (float)(1u << p.mesh_level);
    std::vector<V3d> rest;
    std::vector<V3f> pos;
    std::vector<bool> held;
    rest.reserve(sphere.size());
    pos.reserve(sphere.size());
    for (const V3f& s : sphere) {
        V3f t1 = any_orthonormal(s);
        V3f t2 = cross(s, t1);
        float r1 = (float)rng.next() - 0.5f;
        V3f a = t1 * r1;
        float r2 = (float)rng.next() - 0.5f;
        V3f b = t2 * r2;
        V3f j = ((a + b) * edge_angle) * 0.4f;
        V3d dir = widen(normalize(s + j));
        rest.push_back(dir * rest_r);
        double angle = std::acos(std::clamp(-dir.y, -1.0, 1.0));
        double az = std::atan2(dir.z, dir.x);
        double r, z;
        if (angle <= profile.neck_angle) {
            auto pl = profile.place(angle);
            r = pl.first;
            z = pl.second;
        } else {
            double f = (angle - profile.neck_angle) / (PI - profile.neck_angle);
            r = profile.neck_r * (1.0 - f);
            z = profile.z_neck + 0.5 * profile.neck_r * f;
        }
        held.push_back(angle > profile.neck_angle);
        pos.push_back({(float)(r * std::cos(az)), (float)(bottom_y + z), (float)(r * std::sin(az))});
    }

    std::vector<double> vmass(pos.size(), 0.0);
    std::vector<GpuTri> tris;
    tris.reserve(faces.size());
    for (auto& f : faces) {
        {
            V3d a = rest[f[0]], b = rest[f[1]], c = rest[f[2]];
            if (dot(cross(b - a, c - a), a + b + c) < 0.0) std::swap(f[1], f[2]);
        }
        V3d a = rest[f[0]], b = rest[f[1]], c = rest[f[2]];
        V3d e1 = b - a, e2 = c - a;
        V3d u = normalize(e1);
        V3d w = cross(normalize(cross(e1, e2)), u);
        double m00 = dot(e1, u), m01 = dot(e2, u), m10 = dot(e1, w), m11 = dot(e2, w);
        double det = m00 * m11 - m01 * m10;
        double area = 0.5 * std::fabs(det);
        for (uint32_t vi : f) vmass[vi] += RHO_RUBBER * t0 * area / 3.0;
        GpuTri t;
        t.v[0] = f[0];
        t.v[1] = f[1];
        t.v[2] = f[2];
        t.rest_area = (float)area;
        t.dm_inv[0] = (float)(m11 / det);
        t.dm_inv[1] = (float)(-m01 / det);
        t.dm_inv[2] = (float)(-m10 / det);
        t.dm_inv[3] = (float)(m00 / det);
        tris.push_back(t);
    }
    out.mem_mass.resize(pos.size());
    for (size_t i = 0; i < pos.size(); i++) out.mem_mass[i] = held[i] ? 0.0f : (float)vmass[i];
    out.mem_pos.resize(pos.size());
    for (size_t i = 0; i < pos.size(); i++) out.mem_pos[i] = {pos[i].x, pos[i].y, pos[i].z, 0.0f};

    std::vector<std::vector<uint32_t>> vt(pos.size());
    for (uint32_t ti = 0; ti < tris.size(); ti++)
        for (uint32_t k = 0; k < 3; k++) vt[tris[ti].v[k]].push_back(ti);
    out.vtri_off.assign(1, 0u);
    out.vtri.clear();
    for (auto& l : vt) {
        out.vtri.insert(out.vtri.end(), l.begin(), l.end());
        out.vtri_off.push_back((uint32_t)out.vtri.size());
    }

    // Water particles fill the membrane on a jittered lattice, src/balloon.rs:419-445.
    double spacing = d / (double)std::max<uint32_t>(p.resolution, 16);
    int n = (int)std::ceil(2.0 * radius_max / spacing) + 2;
    int nz = (int)std::ceil(profile.z_neck / spacing) + 1;
    out.particles.clear();
    for (int iy = 0; iy < nz; iy++) {
        double zl = ((double)iy + 0.5) * spacing;
        if (zl > profile.z_neck - spacing) break;
        double rmax = profile.r_at(zl) - 0.5 * spacing;
        if (rmax <= 0.0) continue;
        for (int ix = -n / 2; ix <= n / 2; ix++) {
            for (int iz = -n / 2; iz <= n / 2; iz++) {
                double x = ((double)ix + 0.5 * (double)(iy % 2)) * spacing;
                double z = ((double)iz + 0.5 * (double)(iy % 2)) * spacing;
                double jx = (rng.next() - 0.5) * 0.3 * spacing;
                double jy = (rng.next() - 0.5) * 0.3 * spacing;
                double jz = (rng.next() - 0.5) * 0.3 * spacing;
                if (std::sqrt(x * x + z * z) < rmax)
                    out.particles.push_back({(float)(x + jx), (float)(bottom_y + zl + jy), (float)(z + jz), 1.0f});
            }
        }
    }
    out.profile = std::move(profile);
    out.latex = latex;
    out.bottom_y = bottom_y;
    out.center = center;
    out.knot = knot;
    out.radius_max = radius_max;
    out.spacing = spacing;
    out.tris = std::move(tris);
    return true;
}

// ---- bullets (src/params.rs:155-201, src/flight.rs:41-192, src/bullet.rs) ----------------
enum Nose { ROUND, SPITZER, FLAT, SPHERE };
enum Metal { LEAD, COPPER, STEEL };
struct BulletType {
    const char* name;
    float caliber_mm, mass_g, speed, twist_in;
    Nose nose;
    Metal metal;
    float spin_rpm() const { return twist_in <= 0.0f ? 0.0f : speed / (twist_in * 0.0254f) * 60.0f; }
};
const BulletType BULLETS[7] = {
    {".22 LR, 40 gr lead round nose", 5.7f, 2.59f, 330.0f, 16.0f, ROUND, LEAD},
    {"9 mm Luger, 115 gr FMJ", 9.0f, 7.45f, 360.0f, 10.0f, ROUND, COPPER},
    {".45 ACP, 230 gr FMJ", 11.5f, 14.9f, 255.0f, 16.0f, ROUND, COPPER},
    {"5.56 NATO, 62 gr M855", 5.7f, 4.0f, 940.0f, 7.0f, SPITZER, COPPER},
    {".308 Win, 150 gr spitzer", 7.8f, 9.72f, 860.0f, 10.0f, SPITZER, COPPER},
    {".177 air rifle, 8.4 gr wadcutter", 4.5f, 0.54f, 240.0f, 16.0f, FLAT, LEAD},
    {".177 steel BB", 4.4f, 0.34f, 150.0f, 0.0f, SPHERE, STEEL},
};

double body_share(Nose n) { return n == ROUND ? 0.55 : n == SPITZER ? 0.42 : 1.0; }

constexpr double RHO_AIR_FLIGHT = 1.2;  // src/flight.rs:20

double profile_r(Nose nose, double r, double len, double u) {
    if (nose == SPHERE) return std::sqrt(std::max(r * r - (u - r) * (u - r), 0.0));
    double body = body_share(nose) * len;
    if (u <= body) return r;
    double x = u - body, nl = len - body;
    if (nose == SPITZER) {
        double ro = (r * r + nl * nl) / (2.0 * r);
        return std::max(std::sqrt(std::max(ro * ro - x * x, 0.0)) - (ro - r), 0.0);
    }
    double q = x / nl;
    return r * std::sqrt(std::max(1.0 - q * q, 0.0));
}

constexpr int FLIGHT_SLICES = 24;  // slices of the body in the flight's loads (src/flight.rs:21)

// `Body` of src/flight.rs:78-101. Every u is along the axis from the base.
struct Body {
    Nose nose;
    double radius, length, mass, u_cg, ix, iy;
    double slices[FLIGHT_SLICES][3];  // centre, length and radius of each slice
    double side_area;                 // silhouette area seen from the side
    double u_shoulder, u_cp, u_drag;  // where the cavity leaves the nose; where its lift and drag act
    double cd_water, cd_air, kappa_water, kappa_air;
};

// Miller's twist rule (src/flight.rs:68-76): gyroscopic stability of a bullet of mass m (kg)
// and diameter d (m), l calibres long, one turn per t calibres, at speed v (m/s).
double miller_sg(double m, double d, double l, double t, double v) {
    double grains = m / 64.79891e-6;
    double d_in = d / 0.0254;
    double fps = v / 0.3048;
    return 30.0 * grains / (t * t * (d_in * d_in * d_in) * l * (1.0 + l * l)) * std::cbrt(fps / 2800.0);
}

Body body_new(const ntr_shot& s) {
    Body b;
    b.nose = BULLETS[s.bullet].nose;
    Metal metal = BULLETS[s.bullet].metal;
    double r = 0.5 * (double)s.caliber_mm * 1e-3;
    double mass = (double)s.mass_g * 1e-3;
    double density = metal == LEAD ? 11340.0 : metal == COPPER ? 10500.0 : 7850.0;
    double fill = b.nose == ROUND ? 0.85 : b.nose == SPITZER ? 0.72 : b.nose == FLAT ? 0.95 : 1.0;
    double length = b.nose == SPHERE ? 2.0 * r : mass / density / (PI * r * r) / fill;
    const int fine = 2000;
    double du = length / fine;
    double vol = 0.0, mom = 0.0;
    std::vector<std::pair<double, double>> rad(fine);
    for (int i = 0; i < fine; i++) {
        double u = ((double)i + 0.5) * du;
        rad[i] = {u, profile_r(b.nose, r, length, u)};
    }
    for (auto& q : rad) vol += PI * q.second * q.second * du;
    for (auto& q : rad) mom += PI * q.second * q.second * du * q.first;
    double u_cg = mom / vol;
    double rho = mass / vol;
    double ix = 0.0, iy = 0.0;
    for (auto& q : rad) {
        double r2 = q.second * q.second;
        ix += rho * PI * (r2 * r2) / 2.0 * du;
    }
    for (auto& q : rad) {
        double dd = q.first - u_cg;
        iy += rho * PI * q.second * q.second * du * (q.second * q.second / 4.0 + dd * dd);
    }
    b.radius = r;
    b.length = length;
    b.mass = mass;
    b.u_cg = u_cg;
    b.ix = ix;
    b.iy = iy;
    // The aerodynamic constants of src/flight.rs:133-169.
    const double body = body_share(b.nose) * length;
    double v_nose = 0.0;
    for (auto& q : rad)
        if (q.first > body) v_nose += PI * q.second * q.second * du;
    b.u_cp = b.nose == SPHERE ? r : body + v_nose / (PI * r * r);
    switch (b.nose) {
        case SPITZER: b.u_shoulder = body, b.u_drag = b.u_cp; break;
        case ROUND: b.u_shoulder = body, b.u_drag = length - r * r / (length - body); break;
        case FLAT: b.u_shoulder = length, b.u_drag = length; break;
        default: b.u_shoulder = r, b.u_drag = r; break;
    }
    b.cd_water = (b.nose == ROUND || b.nose == SPHERE) ? 0.30 : b.nose == SPITZER ? 0.20 : 0.82;
    b.cd_air = (b.nose == ROUND || b.nose == SPITZER) ? 0.30 : b.nose == FLAT ? 0.9 : 0.47;
    b.kappa_water = b.nose == SPITZER ? 1.0 : 0.0;
    if (b.nose == SPHERE) {
        b.kappa_air = 0.0;
    } else {
        // Scaled so that the stability is Miller's at the shot's speed with one turn in 30 calibres.
        const double v = std::max((double)s.speed, 1.0), d = 2.0 * r, tw = 30.0;
        const double p = TAU * v / (tw * d);
        const double m_alpha = ix * ix * p * p / (4.0 * iy * miller_sg(mass, d, length / d, tw, v));
        b.kappa_air = m_alpha / (RHO_AIR_FLIGHT * PI * r * r * v * v * (b.u_cp - u_cg));
    }
    for (int j = 0; j < FLIGHT_SLICES; j++) {
        const double sdu = length / (double)FLIGHT_SLICES;
        const double u = ((double)j + 0.5) * sdu;
        b.slices[j][0] = u, b.slices[j][1] = sdu, b.slices[j][2] = profile_r(b.nose, r, length, u);
    }
    b.side_area = 0.0;
    for (auto& q : rad) b.side_area += 2.0 * q.second * du;
    return b;
}

constexpr int SLICES = 32;
constexpr int SECTORS = 16;

std::vector<std::pair<double, double>> outline(const Body& b) {
    const int fine = 4000;
    std::vector<std::pair<double, double>> line(fine + 1);
    for (int i = 0; i <= fine; i++) {
        double u = b.length * (double)i / (double)fine;
        line[i] = {u, profile_r(b.nose, b.radius, b.length, u)};
    }
    std::vector<double> s(1, 0.0);
    for (int i = 0; i < fine; i++) s.push_back(s.back() + std::hypot(line[i + 1].first - line[i].first, line[i + 1].second - line[i].second));
    double total = s.back();
    std::vector<std::pair<double, double>> out;
    for (int k = 0; k <= SLICES; k++) {
        double target = total * (double)k / (double)SLICES;
        size_t i = std::partition_point(s.begin(), s.end(), [&](double x) { return x < target; }) - s.begin();
        i = std::clamp<size_t>(i, 1, fine);
        double f = (target - s[i - 1]) / std::max(s[i] - s[i - 1], 1e-15);
        auto a = line[i - 1], c = line[i];
        out.push_back({a.first + (c.first - a.first) * f, a.second + (c.second - a.second) * f});
    }
    return out;
}

struct Patch {
    float p[4];
    float n[4];
};

std::vector<Patch> surface(const Body& b) {
    std::vector<Patch> out;
    auto ring = [&](double u, double r, double radial, double axial, double area) {
        for (int j = 0; j < SECTORS; j++) {
            double phi = ((double)j + 0.5) * TAU / (double)SECTORS;
            double c = std::cos(phi), sn = std::sin(phi);
            Patch pt;
            pt.p[0] = (float)(r * c);
            pt.p[1] = (float)(r * sn);
            pt.p[2] = (float)(u - b.u_cg);
            pt.p[3] = (float)(area / (double)SECTORS);
            pt.n[0] = (float)(radial * c);
            pt.n[1] = (float)(radial * sn);
            pt.n[2] = (float)axial;
            pt.n[3] = 0.0f;
            out.push_back(pt);
        }
    };
    auto ol = outline(b);
    for (size_t i = 0; i + 1 < ol.size(); i++) {
        double ua = ol[i].first, ra = ol[i].second, ub = ol[i + 1].first, rb = ol[i + 1].second;
        double len = std::hypot(ub - ua, rb - ra);
        if (len <= 0.0) continue;
        double r = 0.5 * (ra + rb);
        ring(0.5 * (ua + ub), r, (ub - ua) / len, -(rb - ra) / len, TAU * r * len);
    }
    const double ends[2][2] = {{0.0, -1.0}, {b.length, 1.0}};
    for (auto& e : ends) {
        double r = profile_r(b.nose, b.radius, b.length, e[0]);
        if (r > 1e-9) ring(e[0], 2.0 / 3.0 * r, 0.0, e[1], PI * r * r);
    }
    return out;
}

double hull(const Body& b) {
    double m = 0.0;
    for (auto& q : outline(b)) m = std::max(m, std::hypot(q.first - b.u_cg, q.second));
    return m;
}

// Body-to-world rotation taking +z onto `n`: the half-way quaternion (cross, 1 + dot),
// normalised, with the two singular cases of glam's DQuat::from_rotation_arc.
std::array<double, 4> rotation_arc_z(V3d n) {
    const V3d from{0, 0, 1};
    double one_minus_eps = 1.0 - 2.0 * 2.220446049250313e-16;
    double d = dot(from, n);
    if (d > one_minus_eps) return {0, 0, 0, 1};
    if (d < -one_minus_eps) {
        // Half a turn about the orthonormal vector Duff et al. give for +z: (0, 1, -0).
        double s = std::sin(PI * 0.5), c = std::cos(PI * 0.5);
        return {0.0 * s, 1.0 * s, -0.0 * s, c};
    }
    V3d c = cross(from, n);
    double q[4] = {c.x, c.y, c.z, 1.0 + d};
    double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    double inv = 1.0 / len;
    return {q[0] * inv, q[1] * inv, q[2] * inv, q[3] * inv};
}

constexpr double LOOKAHEAD = 0.05;

// The hand-over from the flight through the air to the simulation (Flight::new and
// Flight::handoff, src/flight.rs:404-471, 633-637), with the flight's report at impact.
struct Handoff {
    V3d x, u, n, h;  // where the simulation takes over: centre of mass, velocity, axis, angular momentum
    double roll;
    double t_read;    // when
    double t_hit;     // when the tip reaches the balloon
    double v_impact;  // the speed there
    double sg_air;    // gyroscopic stability at impact (infinite for a ball)
    double yaw_impact;  // yaw at impact, rad
    double twist;       // rifling turns per metre
    V3d muzzle_x, muzzle_u;  // the launch that lands on the target
};

// ---- the bullet's flight through still air (src/flight.rs:264-292, 404-676) ------------------
// Rigid body of revolution: state (x, u, n, h, roll), RK4 steps, loads of the leading end and
// of the slices behind it. In still air the reference's water terms have no share (the empty
// field's fill is 0), so only the air terms are restated.
constexpr double CDC_AIR = 1.2, CD_BASE_AIR = 1.17, CF_SKIN = 0.003, CMQ_AIR = -10.0;

struct FState {
    V3d x, u, n, h;
    double roll;
    FState add(const FState& d, double k) const {
        return {x + d.x * k, u + d.u * k, n + d.n * k, h + d.h * k, roll + d.roll * k};
    }
    FState lerp(const FState& o, double k) const {
        FState s = add(o.add(*this, -1.0), k);
        s.n = normalize(s.n);
        return s;
    }
    double yaw() const {
        const double l = length(u);
        const double r = 1.0 / l;
        const V3d uh = (std::isfinite(r) && r > 0.0) ? u * r : V3d{0.0, 0.0, 0.0};
        return std::acos(std::clamp(dot(n, uh), -1.0, 1.0));
    }
};

static inline V3d vdiv(V3d a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline V3d normalize_or(V3d a, V3d fallback) {
    const double r = 1.0 / std::sqrt(dot(a, a));
    return (std::isfinite(r) && r > 0.0) ? a * r : fallback;
}

struct Flight {
    Body b;
    V3d gravity;
    // Force and torque on the body in still air (src/flight.rs:486-598 with an empty field).
    void loads(const FState& s, V3d& force, V3d& torque) const {
        const V3d n = s.n;
        const double p = dot(s.h, n) / b.ix;
        const V3d w_perp = vdiv(s.h - n * dot(s.h, n), b.iy);
        auto at = [&](double u) { return s.x + n * (u - b.u_cg); };
        const double speed = std::max(length(s.u), 1e-6);
        const V3d uhat = vdiv(s.u, speed);
        const double cos_d = std::clamp(dot(n, uhat), -1.0, 1.0);
        const bool nose_first = cos_d >= 0.0;
        const double area = PI * b.radius * b.radius;
        const double rho = RHO_AIR_FLIGHT;
        force = gravity * b.mass;
        torque = {0.0, 0.0, 0.0};
        // The leading end.
        const V3d lead = at(nose_first ? b.length : 0.0);
        const V3d w = s.u + cross(w_perp, lead - s.x);
        const double wl = length(w);
        if (wl >= 1e-9) {
            const double wn = dot(w, n);
            auto axial = [&](double cd) { return n * (-0.5 * rho * cd * area * wn * std::fabs(wn)); };
            V3d f[2] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
            double fu[2] = {0.0, 0.0};
            int nf = 1;
            if (!nose_first) {
                f[0] = axial(CD_BASE_AIR), fu[0] = 0.0;
            } else if (b.nose == FLAT) {
                f[0] = axial(b.cd_air), fu[0] = b.length;
            } else if (b.nose == SPHERE) {
                f[0] = w * (-0.5 * rho * b.cd_air * area * wl), fu[0] = b.u_drag;
            } else {
                const double c = wn / wl;
                f[0] = w * (-0.5 * rho * b.cd_air * area * c * c * wl), fu[0] = b.u_cg;
                f[1] = (w - n * wn) * (-rho * area * b.kappa_air * wn), fu[1] = b.u_cp;
                nf = 2;
            }
            for (int i = 0; i < nf; i++) {
                force = force + f[i] * 1.0;
                torque = torque + cross(at(fu[i]) - s.x, f[i]) * 1.0;
            }
        }
        // The slices: cross-flow drag, Magnus lift, skin friction of the spin.
        for (int j = 0; j < FLIGHT_SLICES; j++) {
            const double u = b.slices[j][0], du = b.slices[j][1], r = b.slices[j][2];
            const V3d xj = at(u);
            const V3d wj = s.u + cross(w_perp, xj - s.x);
            const double wa = dot(wj, n);
            const V3d wc = wj - n * wa;
            const double wcl = length(wc);
            V3d f{0.0, 0.0, 0.0};
            if (b.nose != SPHERE) f = f - wc * (0.5 * rho * CDC_AIR * 2.0 * r * du * wcl);
            if (wcl > 1e-9 && p != 0.0) f = f + cross(n, wc) * (rho * r * r * p * du * std::min(wcl / (r * std::fabs(p)), 1.0));
            const double spin = -0.5 * rho * CF_SKIN * (p * r) * std::fabs(p * r) * TAU * r * du * r;
            force = force + f * 1.0;
            torque = torque + (cross(xj - s.x, f) + n * spin) * 1.0;
        }
        // Pitch damping.
        torque = torque + w_perp * (0.5 * RHO_AIR_FLIGHT * speed * area * 4.0 * b.radius * b.radius * CMQ_AIR * 1.0);
    }
    FState deriv(const FState& s) const {
        V3d f, tq;
        loads(s, f, tq);
        const double p = dot(s.h, s.n) / b.ix;
        const V3d w_perp = vdiv(s.h - s.n * dot(s.h, s.n), b.iy);
        return {s.u, vdiv(f, b.mass), cross(w_perp, s.n), tq, p};
    }
    FState step(const FState& s, double dt) const {
        const FState k1 = deriv(s);
        const FState k2 = deriv(s.add(k1, 0.5 * dt));
        const FState k3 = deriv(s.add(k2, 0.5 * dt));
        const FState k4 = deriv(s.add(k3, dt));
        FState o = s.add(k1, dt / 6.0).add(k2, dt / 3.0).add(k3, dt / 3.0).add(k4, dt / 6.0);
        o.n = normalize(o.n);
        return o;
    }
    // A twentieth of a radian per step at the fastest rotation (src/flight.rs:618-631), in air.
    double dt_of(const FState& s) const {
        const double speed = std::max(length(s.u), 1.0);
        const double p = dot(s.h, s.n) / b.ix;
        const double tumble = length(vdiv(s.h - s.n * dot(s.h, s.n), b.iy));
        const double rho = RHO_AIR_FLIGHT + 0.0 * RHO_WATER;
        const double pull = std::sqrt(rho * PI * b.radius * b.radius * speed * speed * b.length / b.iy);
        return std::min(0.05 / (tumble + b.ix * std::fabs(p) / b.iy + pull), 0.02 / speed);
    }
    V3d tip(const FState& s) const { return s.x + s.n * (b.length - b.u_cg); }
    // Flies until g turns non-negative; the state and time where it crossed zero.
    template <class G>
    std::pair<FState, double> fly(FState s, double t, G g) const {
        double gv = g(s);
        for (int it = 0; it < 2000000; it++) {
            if (gv >= 0.0) break;
            const double dt = dt_of(s);
            const FState next = step(s, dt);
            const double gn = g(next);
            if (gn >= 0.0) {
                const double k = -gv / (gn - gv);
                return {s.lerp(next, k), t + dt * k};
            }
            s = next;
            t += dt;
            gv = gn;
        }
        return {s, t};
    }
};

// Flight::new (src/flight.rs:404-471): aims the bullet from the muzzle, range_m up the line of
// fire, so that its tip crosses the target's plane on the line at the shot's speed (eight
// rounds correcting the aim for the drop and drift and the muzzle speed for the drag), then
// flies it to LOOKAHEAD short of that plane, the simulation's start, and on to the plane.
Handoff flight_handoff(const ntr_shot& s, const Body& b, V3d target, V3d dir, double t_hit, double gravity) {
    Flight f{b, V3d{0.0, -gravity, 0.0}};
    const double v_hit = std::max((double)s.speed, 1.0);
    const double p0 = (double)s.spin_rpm / 60.0 * TAU;
    const double yaw = (double)s.muzzle_yaw_deg * (PI / 180.0);
    const double range = std::max((double)s.range_m, 0.5);
    const V3d muzzle = target - dir * range;
    auto launch = [&](V3d aim, double v) {
        const V3d side = normalize_or(V3d{0.0, 1.0, 0.0} - aim * aim.y, V3d{0.0, 0.0, 1.0});
        const V3d n = aim * std::cos(yaw) + side * std::sin(yaw);
        return FState{muzzle - n * (b.length - b.u_cg), aim * v, n, n * (b.ix * p0), 0.0};
    };
    auto crossing = [&](const FState& st) { return dot(f.tip(st) - target, dir); };
    V3d aim = dir;
    double v_m = v_hit;
    for (int it = 0; it < 8; it++) {
        const FState st = f.fly(launch(aim, v_m), 0.0, crossing).first;
        V3d miss = f.tip(st) - target;
        miss = miss - dir * dot(miss, dir);
        aim = normalize(aim - vdiv(miss, range));
        v_m *= v_hit / length(st.u);
        if (length(miss) < 1e-4 && std::fabs(length(st.u) - v_hit) < 0.01 * v_hit) break;
    }
    Handoff o;
    o.twist = p0 / (TAU * v_m);
    const FState start = launch(aim, v_m);
    o.muzzle_x = start.x, o.muzzle_u = start.u;
    const auto [hand, t_hand] = f.fly(start, 0.0, [&](const FState& st) { return crossing(st) + LOOKAHEAD; });
    const auto [hit, t_c] = f.fly(hand, t_hand, crossing);
    const double shift = t_hit - t_c;
    o.x = hand.x, o.u = hand.u, o.n = hand.n, o.h = hand.h, o.roll = hand.roll;
    o.t_read = t_hand + shift;
    o.t_hit = t_hit;
    const double v = length(hit.u);
    const double p = dot(hit.h, hit.n) / b.ix;
    const double m_alpha = b.kappa_air * RHO_AIR_FLIGHT * PI * b.radius * b.radius * v * v * (b.u_cp - b.u_cg);
    o.sg_air = m_alpha > 0.0 ? b.ix * b.ix * p * p / (4.0 * b.iy * m_alpha) : std::numeric_limits<double>::infinity();
    o.yaw_impact = hit.yaw();
    o.v_impact = v;
    return o;
}

struct GpuBullet {
    float x[4], v[4], q[4], l[4], shape[4], reach[4];
    uint32_t info[4];
};
static_assert(sizeof(GpuBullet) == 112, "Bullet is 112 bytes");

}  // namespace

bool inflate_profile(double shear, double thick, double rest_r, double volume, double rho_g, ntr_profile& out, std::string& err) {
    Latex latex(shear, thick);
    Profile prof;
    if (!inflate(latex, rest_r, volume, rho_g, prof, err)) return false;
    std::memset(&out, 0, sizeof out);
    out.n_samples = (uint32_t)std::min<size_t>(prof.samples.size(), NTR_PROFILE_SAMPLES);
    out.neck_angle = prof.neck_angle;
    out.z_neck = prof.z_neck;
    out.neck_r = prof.neck_r;
    out.volume = prof.volume;
    out.z_centroid = prof.z_centroid;
    out.stretch = prof.stretch;
    for (auto& s : prof.samples) out.r_max = std::max(out.r_max, s.r);
    for (uint32_t i = 0; i < out.n_samples; i++) {
        out.samples[i][0] = prof.samples[i].angle;
        out.samples[i][1] = prof.samples[i].r;
        out.samples[i][2] = prof.samples[i].z;
    }
    return true;
}

// ---- params (src/params.rs, src/presets.rs) ---------------------------------------------
static void shot_set_bullet(ntr_shot& s, uint32_t k) {
    const BulletType& b = BULLETS[k];
    s.bullet = k;
    s.caliber_mm = b.caliber_mm;
    s.mass_g = b.mass_g;
    s.speed = b.speed;
    s.spin_rpm = b.spin_rpm();
}

static ntr_shot shot_default() {
    ntr_shot s{};
    shot_set_bullet(s, 0);
    s.range_m = 10.0f;
    s.muzzle_yaw_deg = 0.5f;
    return s;
}

void params_default(ntr_sim_params& p) {
    std::memset(&p, 0, sizeof p);
    p.n_shots = 1;
    p.shots[0] = shot_default();
    p.balloon_diameter_cm = 16.0f;
    p.balloon_height = 0.55f;
    p.rubber_modulus_mpa = 0.42f;
    p.rubber_rest_diameter_cm = 6.0f;
    p.rubber_break_stretch = 7.0f;
    p.rubber_thickness_mm = 0.25f;
    p.gravity = 9.81f;
    p.spray_amount = 1.0f;
    p.mist_amount = 1.0f;
    p.resolution = 64;
    p.mesh_level = 6;
    p.dt_max = 1e-3f;
    p.seed = 0;
    p.block_cap = 0;
    p.spray_cap = 1200000;
    p.max_iters = 4096;
    p.solve_tol = 1e-5f;
}

// A copy of the last shot, a quarter turn further round (SimParams::add_shot).
static void add_shot(ntr_sim_params& p) {
    ntr_shot s = p.n_shots > 0 ? p.shots[p.n_shots - 1] : shot_default();
    s.azimuth_deg = std::fmod(s.azimuth_deg + 270.0f, 360.0f) - 180.0f;
    p.shots[p.n_shots++] = s;
}

template <class T>
static bool parse_num(const char* v, T& out) {
    char* end = nullptr;
    if constexpr (std::is_same<T, float>::value) {
        out = std::strtof(v, &end);
    } else if constexpr (std::is_same<T, uint64_t>::value) {
        if (*v == '-') return false;
        out = std::strtoull(v, &end, 10);
    } else {
        if (*v == '-') return false;
        unsigned long long x = std::strtoull(v, &end, 10);
        if (x > 0xffffffffull) return false;
        out = (T)x;
    }
    return end && end != v && *end == 0;
}

bool params_set(ntr_sim_params& p, const char* key_c, const char* v, std::string& err) {
    std::string key = key_c ? key_c : "";
    if (!v) {
        err = "missing value";
        return false;
    }
    size_t idx = 0;
    std::string name = key;
    if (key.rfind("shot", 0) == 0) {
        size_t dot = key.find('.');
        if (dot != std::string::npos) {
            uint32_t n = 0;
            if (!parse_num(key.substr(4, dot - 4).c_str(), n)) {
                err = "bad value '" + key.substr(4, dot - 4) + "'";
                return false;
            }
            if (n == 0) {
                err = "shots count from 1";
                return false;
            }
            idx = n - 1;
            name = key.substr(dot + 1);
        }
    }
    if (idx >= NTR_MAX_SHOTS) {
        err = "at most 4 shots";
        return false;
    }
    size_t count = std::max<size_t>(p.n_shots, idx + 1);
    if (name == "shots") {
        uint32_t c = 0;
        if (!parse_num(v, c)) {
            err = std::string("bad value '") + v + "'";
            return false;
        }
        count = c;
    }
    if (count < 1 || count > NTR_MAX_SHOTS) {
        err = "shots 1..4";
        return false;
    }
    ntr_sim_params q = p;
    if (q.n_shots > count) q.n_shots = (uint32_t)count;
    while (q.n_shots < count) add_shot(q);
    ntr_shot& s = q.shots[idx];
    auto bad = [&]() {
        err = std::string("bad value '") + v + "'";
        return false;
    };
    auto setf = [&](float& dst) { return parse_num(v, dst) ? true : bad(); };
    auto setu = [&](uint32_t& dst) { return parse_num(v, dst) ? true : bad(); };
    bool ok = true;
    if (name == "shots") {
    } else if (name == "bullet") {
        uint32_t k = 0;
        if (!parse_num(v, k)) return bad();
        if (k >= 7) {
            err = "bullet 0..6";
            return false;
        }
        shot_set_bullet(s, k);
    } else if (name == "bullet_speed") ok = setf(s.speed);
    else if (name == "caliber") ok = setf(s.caliber_mm);
    else if (name == "mass") ok = setf(s.mass_g);
    else if (name == "spin") ok = setf(s.spin_rpm);
    else if (name == "range") ok = setf(s.range_m);
    else if (name == "yaw") ok = setf(s.muzzle_yaw_deg);
    else if (name == "azimuth") ok = setf(s.azimuth_deg);
    else if (name == "elevation") ok = setf(s.elevation_deg);
    else if (name == "impact_offset") ok = setf(s.impact_offset_cm);
    else if (name == "impact_side") ok = setf(s.impact_side_cm);
    else if (name == "delay") ok = setf(s.delay_ms);
    else if (name == "diameter") ok = setf(q.balloon_diameter_cm);
    else if (name == "height") ok = setf(q.balloon_height);
    else if (name == "modulus") ok = setf(q.rubber_modulus_mpa);
    else if (name == "rest_diameter") ok = setf(q.rubber_rest_diameter_cm);
    else if (name == "break_stretch") ok = setf(q.rubber_break_stretch);
    else if (name == "thickness") ok = setf(q.rubber_thickness_mm);
    else if (name == "gravity") ok = setf(q.gravity);
    else if (name == "spray") ok = setf(q.spray_amount);
    else if (name == "mist") ok = setf(q.mist_amount);
    else if (name == "resolution") ok = setu(q.resolution);
    else if (name == "mesh_level") {
        ok = setu(q.mesh_level);
        if (ok && q.mesh_level > 8) {
            err = "mesh_level 0..8";
            return false;
        }
    } else if (name == "dt_max") ok = setf(q.dt_max);
    else if (name == "seed") {
        ok = parse_num(v, q.seed) ? true : bad();
    } else if (name == "block_cap") ok = setu(q.block_cap);
    else if (name == "spray_cap") ok = setu(q.spray_cap);
    else if (name == "max_iters") ok = setu(q.max_iters);
    else if (name == "solve_tol") ok = setf(q.solve_tol);
    else if (name == "sun" || name == "sky" || name == "env_rotation" || name == "exposure" || name == "dof" ||
             name == "fstop" || name == "focal" || name == "bloom" || name == "caustics" || name == "mist_render" ||
             name == "shutter" || name == "max_bounces" || name == "color") {
        // Renderer-only look parameters: accepted, no effect on the simulation.
    } else {
        err = "unknown parameter '" + key + "'";
        return false;
    }
    if (!ok) return false;
    p = q;
    return true;
}

static bool ieq(const char* a, const char* b) {
    for (; *a && *b; a++, b++)
        if (std::tolower((unsigned char)*a) != std::tolower((unsigned char)*b)) return false;
    return *a == 0 && *b == 0;
}

bool params_preset(ntr_sim_params& p, const char* name, std::string& err) {
    ntr_sim_params q;
    params_default(q);
    auto with_bullet = [](uint32_t k) {
        ntr_shot s = shot_default();
        shot_set_bullet(s, k);
        return s;
    };
    if (ieq(name, "Backlit")) {
    } else if (ieq(name, "Tumbling rifle round")) {
        q.shots[0] = with_bullet(3);
        q.shots[0].speed = 500.0f;
        q.balloon_diameter_cm = 22.0f;
        q.rubber_rest_diameter_cm = 8.0f;
        q.rubber_thickness_mm = 0.5f;
    } else if (ieq(name, "Crossfire")) {
        q.n_shots = 2;
        q.shots[0] = shot_default();
        q.shots[0].impact_offset_cm = 1.5f;
        q.shots[1] = shot_default();
        q.shots[1].azimuth_deg = 90.0f;
        q.shots[1].impact_offset_cm = -1.5f;
    } else if (ieq(name, "Four sides")) {
        const float ad[4][2] = {{0.0f, 0.0f}, {90.0f, 0.5f}, {-180.0f, 1.0f}, {-90.0f, 1.5f}};
        q.n_shots = 4;
        for (int i = 0; i < 4; i++) {
            q.shots[i] = shot_default();
            q.shots[i].azimuth_deg = ad[i][0];
            q.shots[i].delay_ms = ad[i][1];
        }
    } else if (ieq(name, "Moon gravity")) {
        q.gravity = 1.62f;
        q.balloon_diameter_cm = 20.0f;
    } else if (ieq(name, "Weightless")) {
        q.gravity = 0.0f;
    } else if (ieq(name, "Slow pellet")) {
        q.shots[0] = with_bullet(5);
        q.shots[0].speed = 120.0f;
        q.balloon_diameter_cm = 12.0f;
        q.rubber_rest_diameter_cm = 3.2f;
    } else if (ieq(name, "Bounce")) {
        q.shots[0] = with_bullet(6);
        q.shots[0].speed = 40.0f;
        q.rubber_thickness_mm = 1.5f;
        q.rubber_modulus_mpa = 4.0f;
    } else {
        err = std::string("no preset '") + name +
              "', try one of: Backlit, Tumbling rifle round, Crossfire, Four sides, Moon gravity, Weightless, Slow pellet, Bounce";
        return false;
    }
    p = q;
    return true;
}

uint32_t substeps_for(float dt, float sub_dt) {
    float n = std::ceil(1.1f * dt / sub_dt);
    if (!std::isfinite(n)) return 2;
    uint32_t k = n <= 0.0f ? 0u : (n >= 4294967296.0f ? 0xffffffffu : (uint32_t)n);
    k = std::clamp<uint32_t>(k, 2, 256);
    return (k + 1) / 2 * 2;
}

void adapt_after_batch(ntr_world_header& h, const ntr_state& s) {
    h.unconverged += s.unconverged;
    uint32_t mx = h.max_iters ? h.max_iters : 4096;
    if (s.unconverged > 0)
        h.iters = std::min(h.iters * 2, mx);
    else if (s.iters_max > 0)
        h.iters = std::clamp(s.iters_max + s.iters_max / 4 + 2, std::min(8u, mx), mx);
    h.substeps = substeps_for(s.dt_flow, s.mem_dt_seen);
    h.air_substeps = substeps_for(s.dt_flow, s.air_dt_seen);
}

// ---- the world ---------------------------------------------------------------------------
SectionShape section_shape(const ntr_world_header& h, int sec) {
    size_t cells_prev = (size_t)h.n_blocks_prev * 64;
    switch (sec) {
        case NTR_SEC_PARTICLES: return {80, h.n_particles};
        case NTR_SEC_MEM_X: return {16, h.n_verts};
        case NTR_SEC_MEM_V: return {16, h.n_verts};
        case NTR_SEC_MEM_MASS: return {4, h.n_verts};
        case NTR_SEC_MEM_WATER: return {16, h.n_verts};
        case NTR_SEC_MEM_LAYER: return {16 * NTR_LAYER_MODES, h.n_verts};
        case NTR_SEC_MEM_PUSH: return {8, h.n_verts};
        case NTR_SEC_TRIS: return {32, h.n_tris};
        case NTR_SEC_ALIVE: return {4, h.n_tris};
        case NTR_SEC_VTRI_OFF: return {4, (size_t)h.n_verts + 1};
        case NTR_SEC_VTRI: return {4, h.n_vtri};
        case NTR_SEC_BULLETS: return {112, NTR_MAX_SHOTS};
        case NTR_SEC_PATCHES: return {32, NTR_MAX_SHOTS * NTR_MAX_PATCHES};
        case NTR_SEC_OUTLINES: return {8, NTR_MAX_SHOTS * NTR_OUTLINE};
        case NTR_SEC_SECTIONS: return {48, NTR_MAX_SHOTS * NTR_N_SEC};
        case NTR_SEC_BULLET_HIT: return {4, NTR_MAX_SHOTS * NTR_HIT_FIELDS};
        case NTR_SEC_POSE_LOG: return {48, NTR_MAX_SHOTS * NTR_LOG_CAP};
        case NTR_SEC_BLOCKS_PREV: return {4, h.n_blocks_prev};
        case NTR_SEC_BLOCK_ACTIVE: return {4, h.n_blocks_prev};
        case NTR_SEC_AIR: return {4, NTR_AIR_FIELDS * cells_prev};
        case NTR_SEC_SPRAY: return {48, h.n_spray};
        case NTR_SEC_LANDED: return {16, h.n_spray};
        case NTR_SEC_TOUCH: return {4, (size_t)h.wet_res * h.wet_res};
    }
    return {0, 0};
}

void World::shape_sections() {
    for (int s = 0; s < NTR_SEC_COUNT; s++) {
        SectionShape sh = section_shape(h, s);
        sec[s].assign(sh.elem * sh.count, 0);  // zeroed whatever the World held before
    }
}

size_t serialize_into(const World& w, void* out) {
    ntr_world_header h = w.h;
    size_t off = (sizeof(ntr_world_header) + 255) & ~size_t(255);
    for (int s = 0; s < NTR_SEC_COUNT; s++) {
        h.offset[s] = off;
        h.bytes[s] = w.sec[s].size();
        off += (w.sec[s].size() + 255) & ~size_t(255);
    }
    if (!out) return off;
    uint8_t* b = static_cast<uint8_t*>(out);
    std::memcpy(b, &h, sizeof h);
    size_t end = sizeof h;  // everything before `end` is written; the gaps are zeroed
    for (int s = 0; s < NTR_SEC_COUNT; s++) {
        std::memset(b + end, 0, h.offset[s] - end);
        if (!w.sec[s].empty()) std::memcpy(b + h.offset[s], w.sec[s].data(), w.sec[s].size());
        end = h.offset[s] + w.sec[s].size();
    }
    std::memset(b + end, 0, off - end);
    return off;
}

std::vector<uint8_t> serialize(const World& w) {
    std::vector<uint8_t> out(serialize_into(w, nullptr));
    serialize_into(w, out.data());
    return out;
}

bool deserialize(const void* blob, size_t len, World& w, std::string& err) {
    if (!blob || len < sizeof(ntr_world_header)) {
        err = "world blob too short";
        return false;
    }
    std::memcpy(&w.h, blob, sizeof(ntr_world_header));
    if (w.h.magic != NTR_WORLD_MAGIC || w.h.version != NTR_WORLD_VERSION) {
        err = "not a world blob of this version";
        return false;
    }
    if (w.h.n_shots > NTR_MAX_SHOTS || w.h.n_blocks_prev > w.h.block_cap || w.h.n_spray > w.h.spray_cap) {
        err = "world blob counts out of range";
        return false;
    }
    const uint8_t* b = (const uint8_t*)blob;
    for (int s = 0; s < NTR_SEC_COUNT; s++) {
        SectionShape sh = section_shape(w.h, s);
        size_t need = sh.elem * sh.count;
        if (w.h.bytes[s] != need || w.h.offset[s] > len || len - w.h.offset[s] < need) {
            char buf[96];
            snprintf(buf, sizeof buf, "world blob section %d has %llu bytes, expected %zu", s, (unsigned long long)w.h.bytes[s], need);
            err = buf;
            return false;
        }
        w.sec[s].assign(b + w.h.offset[s], b + w.h.offset[s] + need);
    }
    // The mesh indexes device arrays: every index must be in range, and a vertex may be in at
    // most NTR_MAX_VALENCE triangles (the rubber substep keeps one bit per triangle of a vertex).
    const uint32_t* off = w.as<uint32_t>(NTR_SEC_VTRI_OFF);
    const uint32_t* vt = w.as<uint32_t>(NTR_SEC_VTRI);
    if (off[0] != 0u || off[w.h.n_verts] != w.h.n_vtri) {
        err = "world blob vertex-triangle offsets out of range";
        return false;
    }
    for (uint32_t i = 0; i < w.h.n_verts; i++)
        if (off[i + 1] < off[i] || off[i + 1] - off[i] > NTR_MAX_VALENCE) {
            err = "world blob vertex in more than " + std::to_string(NTR_MAX_VALENCE) + " triangles, or offsets decreasing";
            return false;
        }
    for (uint32_t k = 0; k < w.h.n_vtri; k++)
        if (vt[k] >= w.h.n_tris) {
            err = "world blob vertex-triangle index out of range";
            return false;
        }
    const uint32_t* tri = w.as<uint32_t>(NTR_SEC_TRIS);
    for (uint32_t t = 0; t < w.h.n_tris; t++)
        if (tri[8 * (size_t)t] >= w.h.n_verts || tri[8 * (size_t)t + 1] >= w.h.n_verts || tri[8 * (size_t)t + 2] >= w.h.n_verts) {
            err = "world blob triangle vertex out of range";
            return false;
        }
    return true;
}

// Each shot's body and its flight to the balloon (src/sim.rs:280-295): the line of fire from
// the azimuth and elevation, aimed at the impact offsets; the target where that line enters the
// balloon (a radius short of the aim when it misses); the tip's arrival the shot's delay after
// the earliest shot's.
static void shot_flights(const ntr_sim_params& p, const Balloon& scene, std::vector<Handoff>& hand, std::vector<Body>& bodies) {
    float first = 3.4028235e38f;
    for (uint32_t k = 0; k < p.n_shots; k++) first = std::min(first, p.shots[k].delay_ms);
    const float RADS = 3.14159265358979323846f / 180.0f;
    hand.assign(p.n_shots, Handoff{});
    bodies.assign(p.n_shots, Body{});
    for (uint32_t k = 0; k < p.n_shots; k++) {
        const ntr_shot& s = p.shots[k];
        float az = s.azimuth_deg * RADS, el = s.elevation_deg * RADS;
        V3f dir{std::cos(az) * std::cos(el), -std::sin(el), std::sin(az) * std::cos(el)};
        V3f side = normalize_or(cross(dir, V3f{0, 1, 0}), V3f{0, 0, 1});
        V3f aim = (scene.center + V3f{0, 1, 0} * (s.impact_offset_cm * 0.01f)) + side * (s.impact_side_cm * 0.01f);
        auto e = scene.entry(aim, dir);
        V3f target = e ? *e : aim - dir * (float)scene.radius_max;
        double t_hit = (double)(s.delay_ms - first) * 1e-3;
        bodies[k] = body_new(s);
        hand[k] = flight_handoff(s, bodies[k], widen(target), widen(dir), t_hit, (double)p.gravity);
    }
}

static bool check_params(const ntr_sim_params& p, std::string& err);

bool flights(const ntr_sim_params& p, std::vector<ntr_flight>& out, std::string& err) {
    if (!check_params(p, err)) return false;
    Balloon scene;
    if (!build_balloon(p, scene, err)) return false;
    std::vector<Handoff> hand;
    std::vector<Body> bodies;
    shot_flights(p, scene, hand, bodies);
    out.assign(p.n_shots, ntr_flight{});
    for (uint32_t k = 0; k < p.n_shots; k++) {
        const Handoff& h = hand[k];
        ntr_flight& f = out[k];
        const V3d* v[6] = {&h.x, &h.u, &h.n, &h.h, &h.muzzle_x, &h.muzzle_u};
        double* d[6] = {f.x, f.u, f.n, f.h, f.muzzle_x, f.muzzle_u};
        for (int i = 0; i < 6; i++) d[i][0] = v[i]->x, d[i][1] = v[i]->y, d[i][2] = v[i]->z;
        f.roll = h.roll, f.t_read = h.t_read, f.t_hit = h.t_hit, f.v_impact = h.v_impact, f.sg_air = h.sg_air;
        f.yaw_impact_deg = h.yaw_impact * (180.0 / PI);
        f.twist = h.twist;
    }
    return true;
}

static bool check_params(const ntr_sim_params& p, std::string& err) {
    if (p.n_shots < 1 || p.n_shots > NTR_MAX_SHOTS) {
        err = "shots 1..4";
        return false;
    }
    for (uint32_t k = 0; k < p.n_shots; k++)
        if (p.shots[k].bullet >= 7) {
            err = "bullet 0..6";
            return false;
        }
    if (!(p.balloon_diameter_cm > 0.0f) || !(p.rubber_rest_diameter_cm > 0.0f) || !(p.rubber_thickness_mm > 0.0f) ||
        !(p.rubber_modulus_mpa > 0.0f) || !(p.dt_max > 0.0f) || p.mesh_level > 8 || p.resolution > 4096) {
        err = "scene parameters out of range";
        return false;
    }
    return true;
}

bool build_world(const ntr_sim_params& p, World& w, std::string& err) {
    if (!check_params(p, err)) return false;
    Balloon scene;
    if (!build_balloon(p, scene, err)) return false;

    const float WET_HALF = 1.2f;
    const uint32_t WET_RES = 1024;
    const float SOUND = 1480.0f, CFL = 0.8f;
    const uint32_t n_particles = (uint32_t)scene.particles.size();
    const uint32_t n_verts = (uint32_t)scene.mem_pos.size();
    const uint32_t n_tris = (uint32_t)scene.tris.size();
    const double dx = 2.0 * scene.spacing;

    // The sparse grid covers everything the water could reach, src/sim.rs:215-226.
    double top = scene.bottom_y + scene.profile.z_top() + 0.6;
    auto mult4 = [](uint32_t x) { return (x + 3) / 4 * 4; };
    uint32_t nxz = mult4((uint32_t)std::ceil(2.0 * (double)WET_HALF / dx));
    uint32_t ny = mult4((uint32_t)std::ceil(top / dx) + 3);
    float half = (float)((double)nxz * 0.5 * dx);
    float origin[3] = {-half, (float)(-3.0 * dx), -half};
    uint32_t block_cap = p.block_cap;
    if (block_cap == 0) block_cap = 65535u;  // MAX_BLOCKS, src/sim.rs:36
    if (block_cap > 65535u) {
        err = "block_cap is at most 65535";
        return false;
    }

    ntr_world_header& h = w.h;
    std::memset(&h, 0, sizeof h);
    h.magic = NTR_WORLD_MAGIC;
    h.version = NTR_WORLD_VERSION;
    h.n_particles = n_particles;
    h.n_verts = n_verts;
    h.n_tris = n_tris;
    h.n_vtri = (uint32_t)scene.vtri.size();
    h.n_shots = p.n_shots;
    h.n_blocks_prev = 0;
    h.n_spray = 0;
    h.wet_res = WET_RES;
    h.spray_cap = p.spray_cap ? p.spray_cap : 1200000u;
    h.block_cap = block_cap;
    h.iters = 64;
    h.substeps = 0;  // 0 = the zero-length measuring substep has not run yet
    h.air_substeps = 0;
    h.unconverged = 0;
    h.started = 0;
    h.max_iters = p.max_iters ? p.max_iters : 4096;
    h.dx = dx;
    w.shape_sections();

    // The sections come zeroed from shape_sections(): each particle needs its position and its
    // alive flag only.
    float* part = w.as<float>(NTR_SEC_PARTICLES);
    for (uint32_t i = 0; i < n_particles; i++) {
        float* a = part + (size_t)i * 20;
        std::memcpy(a, scene.particles[i].data(), 16);
        a[7] = 1.0f;
    }
    std::memcpy(w.as<float>(NTR_SEC_MEM_X), scene.mem_pos.data(), (size_t)n_verts * 16);
    std::memcpy(w.as<float>(NTR_SEC_MEM_MASS), scene.mem_mass.data(), (size_t)n_verts * 4);
    float* mw = w.as<float>(NTR_SEC_MEM_WATER);
    for (uint32_t i = 0; i < n_verts; i++) mw[4 * i + 3] = 1.0f;  // the rubber starts on the water
    std::memcpy(w.as<uint8_t>(NTR_SEC_TRIS), scene.tris.data(), (size_t)n_tris * 32);
    uint32_t* alive = w.as<uint32_t>(NTR_SEC_ALIVE);
    for (uint32_t t = 0; t < n_tris; t++) alive[t] = 1;
    std::memcpy(w.as<uint32_t>(NTR_SEC_VTRI_OFF), scene.vtri_off.data(), scene.vtri_off.size() * 4);
    std::memcpy(w.as<uint32_t>(NTR_SEC_VTRI), scene.vtri.data(), scene.vtri.size() * 4);
    uint32_t* touch = w.as<uint32_t>(NTR_SEC_TOUCH);
    for (size_t i = 0; i < (size_t)WET_RES * WET_RES; i++) touch[i] = 0xffffffffu;

    // Shots, src/sim.rs:280-310.
    std::vector<Handoff> hand;
    std::vector<Body> bodies;
    shot_flights(p, scene, hand, bodies);
    double t_start = 0.0, t0 = 0.0;
    for (auto& hd : hand) {
        t_start = std::min(t_start, hd.t_read - (0.3 - LOOKAHEAD) / hd.v_impact);
        t0 = std::min(t0, hd.t_read);
    }
    GpuBullet* bl = w.as<GpuBullet>(NTR_SEC_BULLETS);
    Patch* pat = w.as<Patch>(NTR_SEC_PATCHES);
    float* ol = w.as<float>(NTR_SEC_OUTLINES);
    for (uint32_t k = 0; k < p.n_shots; k++) {
        const Body& b = bodies[k];
        auto surf = surface(b);
        if (surf.size() > NTR_MAX_PATCHES) {
            err = "bullet surface has too many patches";
            return false;
        }
        std::memcpy(pat + (size_t)k * NTR_MAX_PATCHES, surf.data(), surf.size() * sizeof(Patch));
        auto line = outline(b);
        for (int j = 0; j < NTR_OUTLINE; j++) {
            ol[(k * NTR_OUTLINE + j) * 2 + 0] = (float)(line[j].first - b.u_cg);
            ol[(k * NTR_OUTLINE + j) * 2 + 1] = (float)line[j].second;
        }
        const Handoff& hd = hand[k];
        auto q = rotation_arc_z(normalize(hd.n));
        GpuBullet g{};
        g.x[0] = (float)hd.x.x, g.x[1] = (float)hd.x.y, g.x[2] = (float)hd.x.z, g.x[3] = (float)b.mass;
        g.v[0] = (float)hd.u.x, g.v[1] = (float)hd.u.y, g.v[2] = (float)hd.u.z, g.v[3] = (float)hd.roll;
        for (int c = 0; c < 4; c++) g.q[c] = (float)q[c];
        g.l[0] = (float)hd.h.x, g.l[1] = (float)hd.h.y, g.l[2] = (float)hd.h.z, g.l[3] = (float)length(hd.u);
        g.shape[0] = (float)b.ix, g.shape[1] = (float)b.iy, g.shape[2] = (float)b.length, g.shape[3] = (float)hull(b);
        g.info[0] = (uint32_t)std::llround((hd.t_read - t0) * 1e9);
        g.info[1] = (uint32_t)surf.size();
        g.info[2] = 0;
        g.info[3] = 0;
        bl[k] = g;
    }
    h.t = t_start;
    h.t_start = t_start;
    h.t0 = t0;

    // The uniform, src/sim.rs:428-441.
    ntr_gpu_params& u = h.params;
    u.origin[0] = origin[0], u.origin[1] = origin[1], u.origin[2] = origin[2], u.origin[3] = (float)dx;
    u.dims[0] = nxz, u.dims[1] = ny, u.dims[2] = nxz, u.dims[3] = n_particles;
    u.bdims[0] = nxz / 4, u.bdims[1] = ny / 4, u.bdims[2] = nxz / 4, u.bdims[3] = block_cap;
    u.gravity[0] = 0.0f, u.gravity[1] = -p.gravity, u.gravity[2] = 0.0f, u.gravity[3] = SOUND;
    u.fluid[0] = (float)RHO_WATER, u.fluid[1] = CFL, u.fluid[2] = p.dt_max, u.fluid[3] = (float)scene.spacing;
    u.wet[0] = WET_HALF;
    u.limits[0] = WET_RES, u.limits[1] = h.spray_cap, u.limits[2] = 0, u.limits[3] = 0;
    u.solve[0] = p.solve_tol > 0.0f ? p.solve_tol : 1e-5f;
    u.mem[0] = n_verts, u.mem[1] = 2, u.mem[2] = 2, u.mem[3] = p.n_shots;
    u.rubber[0] = (float)scene.latex.mu[0], u.rubber[1] = (float)scene.latex.mu[1], u.rubber[2] = (float)scene.latex.mu[2];
    u.rubber[3] = (float)scene.latex.thickness;
    u.rubber2[0] = 0.8f, u.rubber2[1] = p.rubber_break_stretch;
    u.knot[0] = 0.0f, u.knot[1] = (float)(scene.bottom_y + scene.profile.z_neck), u.knot[2] = 0.0f;
    u.knot[3] = (float)scene.profile.neck_r;

    // Nothing limits the first step until the rubber has measured itself; the air starts
    // still at the stable substep of air.wgsl, src/sim.rs:238-241.
    ntr_state& st = h.state;
    std::memset(&st, 0, sizeof st);
    float c_air = std::sqrt(1.4f * 101325.0f / 1.204f);
    st.mem_dt = 3.4028235e38f;
    st.cap_dt = 3.4028235e38f;
    st.air_dt = 0.9f * (float)dx / (3.0f * c_air);
    return true;
}

}  // namespace ntr
