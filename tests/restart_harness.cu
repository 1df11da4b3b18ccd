// CPU check of the restart.dat reader and writer (restart.cu), built by
// tests/test_restart_reader.py: round trip, damaged counts, truncation, and a file
// written by the Python oracle.  No CUDA call is made.
#include "../nrg-mpi_b200/csrc/internal.hpp"
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>
static char g_msg[512];
void nrg_set_error_message(const char* fmt, ...) {
    va_list ap; va_start(ap, fmt); vsnprintf(g_msg, sizeof g_msg, fmt, ap); va_end(ap);
}
using namespace nrg;
static std::vector<char> slurp(const char* p) {
    FILE* f = fopen(p, "rb"); std::vector<char> b; int c;
    while ((c = fgetc(f)) != EOF) b.push_back((char)c);
    fclose(f); return b;
}
static void dump(const char* p, const std::vector<char>& b) { FILE* f = fopen(p, "wb"); fwrite(b.data(), 1, b.size(), f); fclose(f); }
int main(int argc, char** argv) {
    int fails = 0;
    // ---- synthetic round trip
    Model M; M.nIter = 3; M.first = -1; M.nVar = 2; M.nMat = 2; M.nCM = 2; M.nChain = 1; M.nOps = 4;
    M.cb[0] = 1; M.cb[1] = 1; M.cb[2] = 2; M.cb[3] = 2; M.nCoef = 8; M.nBCS = 0; M.flag_spectrum = 1; M.flag_BCS = 0;
    const int nIt = 5, rs = 5, rsf = 8, nbin = 17, nb0 = 4;
    std::mt19937 g(5);
    std::vector<std::vector<int>> si(nIt), bi(nIt), bo(nIt);
    std::vector<std::vector<double>> E(nIt), V(nIt), ims(nIt);
    std::vector<RestoreView> its(nIt);
    for (int x = 0; x < nIt; ++x) {
        const int nsub = 2 + g() % 4, nbf = 6 + g() % 10, nb = 1 + g() % nbf; const long long nv = 10 + g() % 50;
        si[x].resize(nsub * rs); bi[x].resize(nbf * rs); bo[x].resize(nbf * rs);
        for (auto& v : si[x]) v = (int)(g() % 100) - 50;
        for (auto& v : bi[x]) v = (int)(g() % 100) - 50;
        for (auto& v : bo[x]) v = (int)(g() % 100) - 50;
        E[x].resize(nbf); for (auto& v : E[x]) v = (g() % 1000) * 1e-3;
        V[x].resize(nv); for (auto& v : V[x]) v = (g() % 1000) * 1e-3 - 0.5;
        ims[x].resize((size_t)nb * nb * M.nMat); for (auto& v : ims[x]) v = (g() % 1000) * 1e-3;
        RestoreView& R = its[x];
        R.si = si[x].data(); R.bi = bi[x].data(); R.bo = bo[x].data(); R.E = E[x].data(); R.V = V[x].data();
        R.ims = (M.first + x < M.nIter) ? ims[x].data() : nullptr; R.nV = nv; R.nb = nb; R.nb_full = nbf; R.nsub = nsub;
    }
    std::vector<double> ims0(nb0 * nb0 * M.nMat, 0.25), rdm(23, 0.5), bp(2 * nbin * M.nMat, 1.5), bn(2 * nbin * M.nMat, -1.5);
    std::vector<int> fsi(3 * rsf, 7), map(M.nIter + 2, 0);
    int32_t hami[20]; restart_hami(M, 9, 1, true, hami);
    const char* path = "rst_synth.dat";
    if (restart_save(path, M, 2, hami, its, nb0, ims0.data(), rdm.data(), (long long)rdm.size(), fsi.data(), 3, map.data(), bp.data(), bn.data(), nbin) != NRG_OK) { printf("save failed %s\n", g_msg); return 1; }
    RestartData D;
    int rc = restart_load(path, M, nbin, &D);
    bool ok = rc == NRG_OK && D.iteration == 2 && D.rdm == rdm && D.fsi == fsi && D.binPos == bp && D.binNeg == bn && D.ims0 == ims0;
    for (int x = 0; ok && x < nIt; ++x) {
        const RestoreView& A = D.its[x]; const RestoreView& B = its[x];
        ok = A.nb == B.nb && A.nb_full == B.nb_full && A.nsub == B.nsub && A.nV == B.nV &&
             std::equal(A.si, A.si + A.nsub * rs, B.si) && std::equal(A.bi, A.bi + A.nb_full * rs, B.bi) &&
             std::equal(A.bo, A.bo + A.nb_full * rs, B.bo) && std::equal(A.E, A.E + A.nb_full, B.E) &&
             std::equal(A.V, A.V + A.nV, B.V) && (B.ims ? std::equal(A.ims, A.ims + (size_t)A.nb * A.nb * M.nMat, B.ims) : A.ims == nullptr);
    }
    printf("round trip: %s (rc %d %s)\n", ok ? "ok" : "FAIL", rc, rc ? g_msg : ""); fails += !ok;
    // ---- damaged counts: every 4-byte word after the header set to a huge value in turn
    const std::vector<char> good = slurp(path);
    int refused = 0, accepted = 0, crashes = 0;
    for (size_t off = 8 + 80; off + 4 <= good.size(); off += 4) {
        std::vector<char> b = good;
        const int32_t big = 0x7fffffff; memcpy(&b[off], &big, 4);
        dump("rst_bad.dat", b);
        RestartData B2;
        try {
            const int r = restart_load("rst_bad.dat", M, nbin, &B2);
            (r == NRG_OK ? accepted : refused)++;
        } catch (...) { crashes++; }
    }
    printf("huge word at each offset: refused %d, accepted %d (a value word), exceptions %d\n", refused, accepted, crashes);
    fails += crashes > 0;
    // ---- every truncation length is refused
    int trunc_ok = 0, trunc_bad = 0;
    for (size_t len = 0; len < good.size(); len += 7) {
        dump("rst_short.dat", std::vector<char>(good.begin(), good.begin() + len));
        RestartData B3;
        (restart_load("rst_short.dat", M, nbin, &B3) == NRG_OK ? trunc_bad : trunc_ok)++;
    }
    printf("truncations refused %d, accepted %d\n", trunc_ok, trunc_bad); fails += trunc_bad > 0;
    // ---- a file the Python oracle wrote: argv = path nIter first nVar nMat nCM nChain nOps nbin
    if (argc == 10) {
        Model O; O.nIter = atoi(argv[2]); O.first = atoi(argv[3]); O.nVar = atoi(argv[4]); O.nMat = atoi(argv[5]);
        O.nCM = atoi(argv[6]); O.nChain = atoi(argv[7]); O.nOps = atoi(argv[8]);
        RestartData Q;
        const int r = restart_load(argv[1], O, atoi(argv[9]), &Q);
        printf("oracle-written file: %s (iteration %d, %zu eigenvector values) %s\n", r == NRG_OK ? "ok" : "FAIL", Q.iteration, Q.V.size(), r ? g_msg : "");
        fails += r != NRG_OK;
    }
    return fails ? 1 : 0;
}
