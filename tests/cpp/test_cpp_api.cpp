// Exercises the C++ host API (include/vsdmo/DMO.hpp) the way the reference's main.cu uses
// DMOMeshTetFactory / DMOTetClass: build, optimize, read qualities back.
#include <cmath>
#include <cstdio>
#include <vector>
#include "vsdmo/DMO.hpp"

int main() {
    const int n = 6, m = n + 1;
    const float h = 1.0f / n;
    std::vector<float> xyz;
    for (int k = 0; k < m; ++k)
        for (int j = 0; j < m; ++j)
            for (int i = 0; i < m; ++i) {
                float dx = 0.f, dy = 0.f, dz = 0.f;
                if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n) {
                    dx = 0.25f * h * std::sin(1.7f * i + 2.3f * j + 0.7f * k);
                    dy = 0.25f * h * std::cos(0.9f * i + 1.1f * j + 3.1f * k);
                    dz = 0.25f * h * std::sin(2.9f * i + 0.3f * j + 1.9f * k);
                }
                xyz.push_back(i * h + dx); xyz.push_back(j * h + dy); xyz.push_back(k * h + dz);
            }
    const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int step[3] = {1, m, m * m};
    std::vector<int> tets;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (auto& p : perm) {
                    int a = (k * m + j) * m + i, b = a + step[p[0]], c = b + step[p[1]], d = c + step[p[2]];
                    // orient positively on the lattice
                    auto P = [&](int v, int ax) { return (float)((ax == 0 ? v % m : ax == 1 ? (v / m) % m : v / (m * m))); };
                    float e[3][3];
                    for (int ax = 0; ax < 3; ++ax) { e[0][ax] = P(b, ax) - P(a, ax); e[1][ax] = P(c, ax) - P(a, ax); e[2][ax] = P(d, ax) - P(a, ax); }
                    float det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) - e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                                e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
                    if (det < 0) std::swap(b, c);
                    tets.insert(tets.end(), {a, b, c, d});
                }
    try {
        auto mesh = DMO::DMOMeshTetFactory::create((int)xyz.size() / 3, (int)tets.size() / 4, xyz.data(), tets.data());
        DMO::DMOTetClass dmo(*mesh, DMO::QualityCriterium::MEAN_RATIO, 0.5f, 5);
        float q0 = dmo.getQuality();
        dmo.displayQualityGPU();
        dmo.optimize();
        float q1 = dmo.getQuality();
        std::vector<int> hist;
        dmo.getQualityHistogram(hist, 10);
        int total = 0;
        for (int c : hist) total += c;
        std::printf("q0=%.6f q1=%.6f done=%d total=%d colours=%d\n", q0, q1, (int)dmo.isDone(), total, mesh->nColorsInner);
        if (!(q1 > q0) || !dmo.isDone() || total != (int)tets.size() / 4) return 1;
        // an error surfaces as an exception carrying the status
        try {
            DMO::DMOTetClass bad(*mesh, DMO::QualityCriterium::RADIUS_RATIO);
            return 2;
        } catch (const DMO::Error& e) {
            if (e.status != VSDMO_E_UNSUPPORTED) return 3;
        }
        // files: write the optimised mesh, read it back through the factory, and a missing file
        // gives nullptr like the reference's factories
        const std::string base = "/tmp/vsdmo_cpp_api_mesh";
        DMO::writeTetgen(base, static_cast<const DMO::DMOMeshTet&>(*mesh));
        auto again = DMO::DMOMeshTetFactory::create(base);
        if (!again || again->nVertices() != mesh->nVertices()) return 5;
        if (again->getVertexPoints(true) != mesh->getVertexPoints(true)) return 6;
        if (DMO::DMOMeshTetFactory::create(base + "_missing") != nullptr) return 7;
        auto surf = DMO::DMOMeshTriFactory::create(*mesh);
        if (!surf || surf->nVertices() != mesh->nVerticesSurf) return 8;
    } catch (const DMO::Error& e) {
        std::printf("error %d: %s\n", (int)e.status, e.what());
        return 4;
    }
    std::printf("cpp api ok\n");
    return 0;
}
