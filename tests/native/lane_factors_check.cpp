// Host check of the factor-set selection of a packed lane (engine.h
// LaneFactors): two-block chains never reach a third set, also when a step
// range starts past the junction (negative switch_t, as the checkpointed
// adjoint's segments do); triblock chains switch at both junctions.
#include <cstdio>
#include "../../polystring_b200/csrc/engine.h"

int main() {
    static const double a = 0, b = 0, c = 0;
    int bad = 0;
    auto expect = [&](const ps::LaneFactors& lf, int t, int want, const char* what) {
        const int got = lf.set(t);
        const double* f = lf.F(t);
        if (got != want || f != lf.eF[want] || f == nullptr) {
            std::printf("FAIL %s t=%d set %d want %d\n", what, t, got, want);
            bad++;
        }
    };
    ps::LaneFactors ab{{&a, &b}, {&a, &b}, 7};
    for (int t = 0; t < 20; t++) expect(ab, t, t < 7 ? 0 : 1, "diblock");
    ps::LaneFactors late{{&a, &b}, {&a, &b}, -5};
    for (int t = 0; t < 20; t++) expect(late, t, 1, "diblock range past the junction");
    ps::LaneFactors zero{{&a, &a}, {&a, &a}, 0};
    for (int t = 0; t < 20; t++) expect(zero, t, 1, "switch at 0");
    ps::LaneFactors abc{{&a, &b, &c}, {&a, &b, &c}, 5, 12};
    for (int t = 0; t < 20; t++) expect(abc, t, t < 5 ? 0 : (t < 12 ? 1 : 2), "triblock");
    std::printf("%s\n", bad ? "failures" : "ok");
    return bad ? 1 : 0;
}
