// Exercises include/sidr_factory.hpp the way the reference's drivers use
// FactoryContext: structs shaped like SimData and PackedTrees, the three
// evaluate methods, results written for the Python test to compare.
//   factory_shim_main <input.bin> <output.bin>
#include <cstdint>
#include <cstdio>
#include <vector>

#define SIDR_FACTORY_THROW
#include "sidr_factory.hpp"

struct SimDataLike {  // the fields of engine/sim_host.hpp's SimData the shim reads
    int n = 0, m = 0, ld = 0;
    double sigma = 0.2, tmax = 0.0;
    std::vector<double> scores, durations, open_t, close_t, dist, dist_to_depot;
};

struct PackedTreesLike {  // engine/factory.cuh's PackedTrees
    std::vector<int32_t> ops, args, offsets, lengths;
};

template <class T>
static void rd(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) throw std::runtime_error("short input");
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[9];
    double tmax;
    if (std::fread(hdr, 4, 9, f) != 9 || std::fread(&tmax, 8, 1, f) != 1) return 2;
    const int n = hdr[0], m = hdr[1], P = hdr[2], T = hdr[3], G = hdr[4], gs = hdr[5], mg = hdr[6],
              nm = hdr[7], nn = hdr[8];
    SimDataLike sd;
    sd.n = n;
    sd.m = m;
    sd.ld = n + 1;
    sd.tmax = tmax;
    std::vector<double> zp, sampled;
    std::vector<int64_t> masks;
    PackedTreesLike pk;
    rd(f, sd.scores, n);
    rd(f, sd.durations, n);
    rd(f, sd.open_t, n);
    rd(f, sd.close_t, n);
    rd(f, sd.dist, (size_t)(n + 1) * (n + 1));
    rd(f, sd.dist_to_depot, n);
    rd(f, zp, 10);
    rd(f, pk.ops, nn);
    rd(f, pk.args, 2 * (size_t)nn);
    rd(f, pk.offsets, P);
    rd(f, pk.lengths, P);
    rd(f, sampled, (size_t)G * T * n);
    rd(f, masks, (size_t)nm * 61);
    std::fclose(f);

    std::vector<double> zp2 = sidr::zp_of_sidr(sd);
    sidr::FactoryContextT<SimDataLike, PackedTreesLike> ctx(sd, zp);
    std::vector<int64_t> mask0(masks.begin(), masks.begin() + 61);
    std::vector<double> first(sampled.begin(), sampled.begin() + (size_t)T * n);
    std::vector<double> a = ctx.evaluate(pk, first, T, mask0);
    std::vector<double> b = ctx.evaluate_grouped(pk, sampled, G, T, gs, mask0);
    std::vector<double> c = ctx.evaluate_grouped_masks(pk, sampled, T, gs, mg, masks);
    FILE* o = std::fopen(argv[2], "wb");
    std::fwrite(zp2.data(), 8, 10, o);
    std::fwrite(a.data(), 8, a.size(), o);
    std::fwrite(b.data(), 8, b.size(), o);
    std::fwrite(c.data(), 8, c.size(), o);
    std::fclose(o);
    return 0;
}
