// Synthetic mesh point generators for the benchmark configurations.
//
// Poisson-disk sampling (Bridson's grid-accelerated dart throwing) in the unit
// disk (radius 1, centred at the origin) or the unit square [0,1]^2.  The RNG is
// a counter-free xoshiro256** seeded through splitmix64, so a seed reproduces
// the same point set on any machine.  Host-only; no CUDA.
//
// Built as a stand-alone program (lib/owtk_meshgen), not a library, so a
// process that only reads its output maps none of this project's code:
//
//     owtk_meshgen <radius> <domain 0|1> <seed> <max_points> <output file>
//
// writes the points as raw little-endian float64 (x, y) pairs and exits 0,
// or exits 2 when more than max_points would be needed, 1 on a usage or I/O
// error.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {

struct Rng {
    std::uint64_t s[4];
    explicit Rng(std::uint64_t seed)
    {
        for (auto& w : s) {
            seed += 0x9e3779b97f4a7c15ULL;
            std::uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            w = z ^ (z >> 31);
        }
    }
    static std::uint64_t rotl(std::uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    std::uint64_t next()
    {
        const std::uint64_t result = rotl(s[1] * 5, 7) * 9;
        const std::uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return result;
    }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
};

}  // namespace

extern "C" {

// domain: 0 = unit square [0,1]^2, 1 = unit disk.  Writes at most max_points
// (x, y) pairs to xy and returns the number written (or -1 if it overflowed).
long long owtk_poisson_disk(double radius, int domain, unsigned long long seed,
                            long long max_points, double* xy)
{
    const double x0 = domain == 1 ? -1.0 : 0.0;
    const double extent = domain == 1 ? 2.0 : 1.0;
    const double cell = radius / std::sqrt(2.0);
    const long long g = static_cast<long long>(std::ceil(extent / cell));
    std::vector<std::int32_t> grid(static_cast<std::size_t>(g * g), -1);
    std::vector<std::int32_t> active;
    active.reserve(1 << 20);
    Rng rng(seed);
    long long count = 0;
    auto inside = [&](double x, double y) {
        if (domain == 1) return x * x + y * y < 1.0;
        return x >= 0.0 && x < 1.0 && y >= 0.0 && y < 1.0;
    };
    auto cell_of = [&](double v) {
        long long c = static_cast<long long>((v - x0) / cell);
        return c < 0 ? 0 : (c >= g ? g - 1 : c);
    };
    auto add = [&](double x, double y) -> bool {
        if (count >= max_points) return false;
        xy[2 * count] = x;
        xy[2 * count + 1] = y;
        grid[static_cast<std::size_t>(cell_of(y) * g + cell_of(x))] = static_cast<std::int32_t>(count);
        active.push_back(static_cast<std::int32_t>(count));
        ++count;
        return true;
    };
    const double r2 = radius * radius;
    add(domain == 1 ? 0.0 : 0.5, domain == 1 ? 0.0 : 0.5);
    const int attempts = 30;
    while (!active.empty()) {
        const std::size_t pick = static_cast<std::size_t>(rng.next() % active.size());
        const std::int32_t p = active[pick];
        const double px = xy[2 * p], py = xy[2 * p + 1];
        bool placed = false;
        for (int a = 0; a < attempts; ++a) {
            const double ang = 2.0 * M_PI * rng.uniform();
            const double rad = radius * std::sqrt(1.0 + 3.0 * rng.uniform());
            const double cx = px + rad * std::cos(ang), cy = py + rad * std::sin(ang);
            if (!inside(cx, cy)) continue;
            const long long gx = cell_of(cx), gy = cell_of(cy);
            bool ok = true;
            for (long long yy = gy - 2; yy <= gy + 2 && ok; ++yy) {
                if (yy < 0 || yy >= g) continue;
                for (long long xx = gx - 2; xx <= gx + 2; ++xx) {
                    if (xx < 0 || xx >= g) continue;
                    const std::int32_t q = grid[static_cast<std::size_t>(yy * g + xx)];
                    if (q < 0) continue;
                    const double dx = xy[2 * q] - cx, dy = xy[2 * q + 1] - cy;
                    if (dx * dx + dy * dy < r2) { ok = false; break; }
                }
            }
            if (ok) {
                if (!add(cx, cy)) return -1;
                placed = true;
                break;
            }
        }
        if (!placed) {
            active[pick] = active.back();
            active.pop_back();
        }
    }
    return count;
}

}  // extern "C"

int main(int argc, char** argv)
{
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s radius domain(0 square, 1 disk) seed max_points output\n", argv[0]);
        return 1;
    }
    const double radius = std::strtod(argv[1], nullptr);
    const int domain = std::atoi(argv[2]);
    const unsigned long long seed = std::strtoull(argv[3], nullptr, 10);
    const long long max_points = std::strtoll(argv[4], nullptr, 10);
    if (!(radius > 0.0) || (domain != 0 && domain != 1) || max_points <= 0) {
        std::fprintf(stderr, "owtk_meshgen: invalid arguments\n");
        return 1;
    }
    std::vector<double> xy(static_cast<std::size_t>(2 * max_points));
    const long long count = owtk_poisson_disk(radius, domain, seed, max_points, xy.data());
    if (count < 0) return 2;
    std::FILE* f = std::fopen(argv[5], "wb");
    if (f == nullptr) return 1;
    const std::size_t want = static_cast<std::size_t>(2 * count);
    const bool ok = std::fwrite(xy.data(), sizeof(double), want, f) == want;
    return (std::fclose(f) == 0 && ok) ? 0 : 1;
}
