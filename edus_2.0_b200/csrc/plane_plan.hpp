// Host-side plan of the in-shared-memory plane FFT (fft_plane.cuh).
//
// Include after <vector>, <string>, <cmath>, <algorithm> and fft_plane.cuh;
// this header includes nothing itself so that a translation unit may place
// it, with fft_plane.cuh, inside an enclosing namespace.
namespace edus {

// Radices with an in-register DFT in fft_plane.cuh.
inline const std::vector<int>& supported_radices() {
    static const std::vector<int> r = {13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
    return r;
}

inline int gcd_int(int a, int b) {
    while (b) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Stage radices of one axis, in DIF order.  Fewest stages first; then the
// last stage (unit stride along the innermost axis: each thread reads R
// consecutive elements) gets the radix whose 16-byte stride shares the fewest
// factors with the 8 slots of a 128-byte shared-memory wavefront; the other
// stages follow in decreasing radix.
inline bool choose_radices(int n, std::vector<int>& best) {
    best.clear();
    if (n == 1) return true;
    std::vector<int> cur;
    std::vector<int> bestset;
    int best_key[2] = {1 << 30, 1 << 30};
    // depth-first over non-increasing radix sequences (multisets)
    struct Rec {
        static void go(int m, int maxr, std::vector<int>& cur, std::vector<int>& bestset, int* best_key) {
            if (m == 1) {
                int gbest = 8;
                for (int r : cur) gbest = std::min(gbest, gcd_int(r, 8));
                const int key0 = (int)cur.size(), key1 = gbest;
                if (key0 < best_key[0] || (key0 == best_key[0] && key1 < best_key[1])) {
                    best_key[0] = key0;
                    best_key[1] = key1;
                    bestset = cur;
                }
                return;
            }
            if ((int)cur.size() >= kMaxStages) return;
            for (int r : supported_radices()) {
                if (r > maxr || m % r) continue;
                cur.push_back(r);
                go(m / r, r, cur, bestset, best_key);
                cur.pop_back();
            }
        }
    };
    Rec::go(n, 1 << 30, cur, bestset, best_key);
    if (bestset.empty()) return false;
    // last stage: the radix with the smallest gcd with 8 (largest on ties)
    int li = 0;
    for (int i = 1; i < (int)bestset.size(); ++i) {
        const int gi = gcd_int(bestset[i], 8), gl = gcd_int(bestset[li], 8);
        if (gi < gl || (gi == gl && bestset[i] > bestset[li])) li = i;
    }
    const int last = bestset[li];
    bestset.erase(bestset.begin() + li);
    std::sort(bestset.begin(), bestset.end(), [](int a, int b) { return a > b; });
    best = bestset;
    best.push_back(last);
    return true;
}

// Frequency index left at each position by the in-place DIF pass.
inline void dif_positions(int n, const std::vector<int>& r, std::vector<int>& freq_at_pos) {
    freq_at_pos.assign(n, 0);
    for (int k = 0; k < n; ++k) {
        int pos = 0, len = n, kk = k;
        for (int radix : r) {
            len /= radix;
            pos += (kk % radix) * len;
            kk /= radix;
        }
        freq_at_pos[pos] = k;
    }
}

struct PlaneTables {
    std::vector<double2> roots;  // per axis exp(-2 pi i j / n)
    std::vector<double> rpos;    // per axis Gamma-centred coordinate of each position
    std::vector<int> fq;         // per axis frequency index of each position
    int fqoff[3] = {0, 0, 0};
};

// Plan for an N0 x N1 x N2 plane; false (with a message) if a size has a
// prime factor without a DFT here.
inline bool build_plane_plan(const int N[3], PlanePlan& plan, PlaneTables& tab, std::string& err) {
    plan = PlanePlan{};
    tab = PlaneTables{};
    int stride = 1;
    for (int ax = 2; ax >= 0; --ax) {
        AxisPlan& A = plan.ax[ax];
        A.n = N[ax];
        A.inner = stride;
        A.fd_inner = make_fastdiv(stride);
        stride *= A.n;
        std::vector<int> r;
        if (!choose_radices(A.n, r)) {
            err = "grid size " + std::to_string(A.n) + " has a prime factor other than 2, 3, 5, 7, 11, 13";
            return false;
        }
        A.nst = (int)r.size();
        int L = A.n;
        for (int s = 0; s < A.nst; ++s) {
            A.r[s] = r[s];
            L /= r[s];
            A.L[s] = L;
            A.fd_nbfly[s] = make_fastdiv(A.n / r[s]);
            A.fd_L[s] = make_fastdiv(L);
        }
        A.rootoff = (int)tab.roots.size();
        for (int j = 0; j < A.n; ++j) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * j / A.n;
            tab.roots.push_back(make_double2((double)cosl(a), (double)sinl(a)));
        }
        A.rposoff = (int)tab.rpos.size();
        std::vector<int> fq;
        dif_positions(A.n, r, fq);
        tab.fqoff[ax] = (int)tab.fq.size();
        for (int q = 0; q < A.n; ++q) {
            const int j = fq[q];
            // Gamma-centred coordinate, [-N/2, N/2) (MeshGrid.cpp:352-375, 458-486)
            tab.rpos.push_back(2 * j >= A.n ? double(j - A.n) : double(j));
            tab.fq.push_back(j);
        }
    }
    plan.Nk = N[0] * N[1] * N[2];
    plan.fd_n1 = make_fastdiv(N[1]);
    plan.fd_n2 = make_fastdiv(N[2]);
    return true;
}

}  // namespace edus
