// Device-resident replay of the reference driver (main.F90:142-252): the forward NRG sweep
// (nrgIteration.F90 -> prepareBasis, diagonalization, postprocess), the backward reduced
// density matrices and the CFS spectrum at T = 0.  Eigenvector blocks, invariant
// matrices, density matrices and bins stay in device memory; the host keeps the integer
// bookkeeping (basis records, sector tables, the truncation decision), which needs the
// eigenvalues of each iteration (one small device-to-host copy per iteration).
#include "internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

using namespace nrg;

namespace {

// sortBasisArray (module.F90:531-602): exchange sort of whole records.  When no two
// records share (basis, reference) any correct sort gives its result; ties are resolved
// by replaying the exchange sequence.
void sort_basis(std::vector<int>& rec, int n, int nVar) {
    const int rs = nVar + 3;
    auto greater = [&](const int* a, const int* b) {
        for (int i = 0; i < nVar; ++i) {
            if (a[i] > b[i]) return true;
            if (a[i] < b[i]) return false;
        }
        return a[nVar] > b[nVar];
    };
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
        return greater(&rec[(size_t)y * rs], &rec[(size_t)x * rs]);
    });
    bool ties = false;
    for (int i = 1; i < n && !ties; ++i) {
        const int* a = &rec[(size_t)idx[i - 1] * rs];
        const int* b = &rec[(size_t)idx[i] * rs];
        ties = !greater(b, a) && !greater(a, b);
    }
    if (!ties) {
        std::vector<int> out((size_t)n * rs);
        for (int i = 0; i < n; ++i) std::memcpy(&out[(size_t)i * rs], &rec[(size_t)idx[i] * rs], sizeof(int) * rs);
        rec.swap(out);
        return;
    }
    std::vector<int> tmp(rs);
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            int* a = &rec[(size_t)i * rs];
            int* b = &rec[(size_t)j * rs];
            if (greater(a, b)) {
                std::memcpy(tmp.data(), a, sizeof(int) * rs);
                std::memcpy(a, b, sizeof(int) * rs);
                std::memcpy(b, tmp.data(), sizeof(int) * rs);
            }
        }
}

struct IterRec {
    int nb_full = 0, nb_kept = 0;
    std::vector<int> kept;
    std::vector<double> Esec;
    std::vector<long long> rdm_off;
};

}  // namespace

extern "C" int nrg_run(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out) {
    if (!ctx || !in) return NRG_ERR_INVALID;
    if (!ctx->model.set) { nrg_set_error_message("nrg_context_set_model has not been called"); return NRG_ERR_STATE; }
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    const Model& M = ctx->model;
    const int nVar = M.nVar, rs = nVar + 3, nOps = M.nOps, first = M.first, nIter = M.nIter;
    const int nIt = nIter - first + 1;
    const bool spectrum = in->spectrum && M.nMat > 0;
    cudaStream_t st = ctx->stream;

    cudaEvent_t ev[4];
    for (auto& e : ev) NRG_CUDA_TRY(cudaEventCreate(&e));
    NRG_CUDA_TRY(cudaEventRecord(ev[0], st));

    // ---- initial state (read_initial_basis) ----
    int nb_old = in->numberOfBasis;
    std::vector<int> bo(in->basis_output, in->basis_output + (size_t)nb_old * rs);
    DevBuf& bEold0 = ctx->slot(3);
    DevBuf& bIM0 = ctx->slot(1);
    NRG_TRY(bEold0.ensure(sizeof(double) * nb_old));
    NRG_TRY(bIM0.ensure(sizeof(double) * (size_t)nb_old * nb_old * M.nCM));
    NRG_CUDA_TRY(cudaMemcpyAsync(bEold0.p, in->eigenvalue, sizeof(double) * nb_old, cudaMemcpyHostToDevice, st));
    NRG_CUDA_TRY(cudaMemcpyAsync(bIM0.p, in->invariant_matrix, sizeof(double) * (size_t)nb_old * nb_old * M.nCM,
                                 cudaMemcpyHostToDevice, st));
    const double* dEold = bEold0.as<double>();
    const double* dIMold = bIM0.as<double>();
    const double* dIMSold = nullptr;
    if (spectrum) {
        DevBuf& b = ctx->slot(9);
        NRG_TRY(b.ensure(sizeof(double) * (size_t)nb_old * nb_old * M.nMat));
        NRG_CUDA_TRY(cudaMemcpyAsync(b.p, in->invariant_matrix_spectrum, sizeof(double) * (size_t)nb_old * nb_old * M.nMat,
                                     cudaMemcpyHostToDevice, st));
        dIMSold = b.as<double>();
    }
    if ((int)ctx->iter_sectors.size() < nIt) ctx->iter_sectors.resize(nIt);
    std::vector<IterRec> recs(nIt);
    int startTrancation = nIter + 1;
    bool flag_truncation = false;
    auto slotV = [&](int idx) -> DevBuf& { return ctx->slot(20 + 3 * (size_t)idx); };
    auto slotE = [&](int idx) -> DevBuf& { return ctx->slot(21 + 3 * (size_t)idx); };
    auto slotS = [&](int idx) -> DevBuf& { return ctx->slot(22 + 3 * (size_t)idx); };

    // ---- forward sweep ----
    for (int it = first; it <= nIter; ++it) {
        const int idx = it - first;
        IterRec& R = recs[idx];
        // prepareBasis (prepareBasis.F90:31-114)
        const int nb = nb_old * nOps;
        std::vector<int> rec((size_t)nb * rs);
        for (int i = 0; i < nb_old; ++i)
            for (int j = 0; j < nOps; ++j) {
                int* r = &rec[((size_t)i * nOps + j) * rs];
                for (int v = 0; v < nVar; ++v) r[v] = bo[(size_t)i * rs + v] - M.op(j, v);
                r[nVar] = i + 1;
                r[nVar + 1] = bo[(size_t)i * rs + nVar];
                r[nVar + 2] = j + 1;
            }
        sort_basis(rec, nb, nVar);
        std::vector<int> si;
        {
            int s0 = 0;
            long long ce = 1;
            for (int i = 1; i <= nb; ++i) {
                bool brk = (i == nb);
                if (!brk)
                    for (int v = 0; v < nVar; ++v)
                        if (rec[(size_t)i * rs + v] != rec[(size_t)s0 * rs + v]) { brk = true; break; }
                if (brk) {
                    const int d = i - s0;
                    for (int v = 0; v < nVar; ++v) si.push_back(rec[(size_t)s0 * rs + v]);
                    si.push_back(d);
                    si.push_back((int)std::min(ce, 0x7fffffffLL));
                    si.push_back(s0 + 1);
                    ce += (long long)d * d;
                    s0 = i;
                }
            }
        }
        const int nsub = (int)(si.size() / rs);
        Sectors& S = ctx->iter_sectors[idx];
        NRG_TRY(S.build(nsub, si.data(), nb, rec.data(), nVar, nOps));
        NRG_TRY(S.upload(st));
        // diagonalization
        DevBuf& bV = slotV(idx);
        DevBuf& bE = slotE(idx);
        NRG_TRY(bV.ensure(sizeof(double) * (size_t)S.sizeV));
        NRG_TRY(bE.ensure(sizeof(double) * (size_t)nb));
        DiagOut dout;
        NRG_TRY(diag_device(ctx, it, S, dEold, nb_old, dIMold, bV.as<double>(), bE.as<double>(), &dout));
        if (out && out->groundStateEnergy) out->groundStateEnergy[idx] = dout.groundStateEnergy;
        R.Esec.resize(nb);
        NRG_CUDA_TRY(cudaMemcpyAsync(R.Esec.data(), bE.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
        NRG_CUDA_TRY(cudaStreamSynchronize(st));
        // postprocess: truncation (postprocess.F90:71-160)
        std::vector<int> order(nb);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return R.Esec[a] < R.Esec[b]; });
        int nbk = nb;
        if (it != first && it != nIter && nb > M.truncation) {
            if (startTrancation > it) { startTrancation = it; flag_truncation = true; }
            const int limit = (int)(M.truncation * 1.2);
            double Ecut = R.Esec[order[M.truncation - 1]];
            int i = M.truncation + 1, cutoff = M.truncation;
            Ecut = Ecut + 0.000001;
            while (i <= nb) {
                if (R.Esec[order[i - 1]] <= Ecut) cutoff++; else break;
                ++i;
            }
            while (cutoff > limit) {
                Ecut = Ecut - 0.001;
                for (int q = cutoff; q >= 1; --q) {
                    if (R.Esec[order[q - 1]] > Ecut) cutoff--; else break;
                }
            }
            nbk = cutoff;
        }
        std::sort(order.begin(), order.begin() + nbk);   // sortByIndex (:140)
        if (out && out->flow && out->flowStride > 0) {
            std::vector<double> e(nbk);
            for (int q = 0; q < nbk; ++q) e[q] = R.Esec[order[q]];
            std::sort(e.begin(), e.end());
            for (int q = 0; q < out->flowStride; ++q)
                out->flow[(size_t)idx * out->flowStride + q] = q < nbk ? e[q] : NAN;
        }
        // basis_output after truncation (:143-160)
        std::vector<int> rowSec(nb);
        for (int s = 0; s < nsub; ++s)
            for (int j = 0; j < S.dim[s]; ++j) rowSec[S.start[s] + j] = s;
        std::vector<int> bo_new((size_t)nb * rs, 0);
        std::vector<double> Eold_next(nbk);
        R.kept.assign(nsub, 0);
        for (int q = 0; q < nb; ++q) {
            const int row = order[q], s = rowSec[row];
            int* r = &bo_new[(size_t)q * rs];
            for (int v = 0; v < nVar; ++v) r[v] = S.qn[(size_t)s * nVar + v];
            r[nVar] = row - S.start[s] + 1;
            if (q < nbk) { Eold_next[q] = R.Esec[row]; R.kept[s]++; }
        }
        R.nb_full = nb;
        R.nb_kept = nbk;
        if (out && out->kept) out->kept[idx] = nbk;
        if (out && out->numberOfBasisFull) out->numberOfBasisFull[idx] = nb;
        // invariant matrices for the next iteration (postprocess.F90:189-204)
        const double* dIMnew = dIMold;
        const double* dIMSnew = dIMSold;
        if (it < nIter) {
            DevBuf& bIM = ctx->slot(1 + ((idx + 1) & 1));
            NRG_TRY(bIM.ensure(sizeof(double) * (size_t)nbk * nbk * M.nCM));
            NRG_TRY(invmat_device(ctx, S, R.kept, bV.as<double>(), bIM.as<double>()));
            dIMnew = bIM.as<double>();
            if (spectrum) {
                DevBuf& bS = slotS(idx);
                NRG_TRY(bS.ensure(sizeof(double) * (size_t)nbk * nbk * M.nMat));
                NRG_TRY(invmat_spec_device(ctx, S, R.kept, bV.as<double>(), nb_old, dIMSold, bS.as<double>()));
                dIMSnew = bS.as<double>();
            }
        }
        DevBuf& bEo = ctx->slot(3 + ((idx + 1) & 1));
        NRG_TRY(bEo.ensure(sizeof(double) * nbk));
        NRG_CUDA_TRY(cudaMemcpyAsync(bEo.p, Eold_next.data(), sizeof(double) * nbk, cudaMemcpyHostToDevice, st));
        NRG_CUDA_TRY(cudaStreamSynchronize(st));
        dEold = bEo.as<double>();
        dIMold = dIMnew;
        dIMSold = dIMSnew;
        bo.swap(bo_new);
        nb_old = nbk;
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[1], st));

    const int nbin = M.numberOfBin();
    const size_t nw = (size_t)nbin * std::max(M.nMat, 1);
    DevBuf& bBins = ctx->slot(6);
    NRG_TRY(bBins.ensure(sizeof(double) * 2 * nw));
    double* dPos = bBins.as<double>();
    double* dNeg = dPos + nw;
    NRG_TRY(run_fill(ctx, dPos, (long long)(2 * nw), 0.0));

    // ---- backward reduced density matrices (initializeReducedDensity, main.F90:188-201) ----
    DevBuf& bRdm = ctx->slot(5);
    const int last = nIter - first;
    if (spectrum && flag_truncation) {
        long long off = 0;
        for (int N = nIter; N >= startTrancation; --N) {
            IterRec& R = recs[N - first];
            R.rdm_off.assign(R.kept.size(), -1);
            for (size_t s = 0; s < R.kept.size(); ++s)
                if (R.kept[s] > 0) { R.rdm_off[s] = off; off += (long long)R.kept[s] * R.kept[s]; }
        }
        NRG_TRY(bRdm.ensure(sizeof(double) * (size_t)std::max(off, 1LL)));
        NRG_TRY(run_fill(ctx, bRdm.as<double>(), off, 0.0));
        // T = 0 seed: projector on the ground states at the last iteration
        IterRec& RL = recs[last];
        const Sectors& SL = ctx->iter_sectors[last];
        int deg = 0;
        for (int i = 0; i < RL.nb_full; ++i) deg += RL.Esec[i] < 1.0e-8;
        const double inv = 1.0 / (double)deg;
        for (int s = 0; s < SL.nsub; ++s)
            for (int p = 0; p < RL.kept[s]; ++p)
                if (RL.Esec[SL.start[s] + p] < 1.0e-8)
                    NRG_CUDA_TRY(cudaMemcpyAsync(bRdm.as<double>() + RL.rdm_off[s] + (long long)p * RL.kept[s] + p, &inv,
                                                 sizeof(double), cudaMemcpyHostToDevice, st));
        NRG_CUDA_TRY(cudaStreamSynchronize(st));
        DevBuf& bTr = ctx->slot(7);
        NRG_TRY(bTr.ensure(sizeof(double) * (size_t)(nIter + 2)));
        for (int N = nIter - 1; N >= startTrancation; --N) {
            IterView P, C;
            const int ip = N - first, ic = N + 1 - first;
            P.S = &ctx->iter_sectors[ip]; P.kept = recs[ip].kept; P.d_V = slotV(ip).as<double>();
            P.d_rdm = bRdm.as<double>(); P.rdm_off = recs[ip].rdm_off;
            C.S = &ctx->iter_sectors[ic]; C.kept = recs[ic].kept; C.d_V = slotV(ic).as<double>();
            C.d_rdm = bRdm.as<double>(); C.rdm_off = recs[ic].rdm_off;
            NRG_TRY(rdm_step_device(ctx, P, C, bRdm.as<double>(), bTr.as<double>() + N));
        }
        if (out && out->rdmTrace) {
            std::vector<double> tr(nIter + 1, NAN);
            NRG_CUDA_TRY(cudaMemcpyAsync(tr.data(), bTr.p, sizeof(double) * (nIter + 1), cudaMemcpyDeviceToHost, st));
            NRG_CUDA_TRY(cudaStreamSynchronize(st));
            for (int N = 0; N <= nIter; ++N) out->rdmTrace[N] = (N >= startTrancation && N < nIter) ? tr[N] : NAN;
        }
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[2], st));

    // ---- CFS spectrum (main.F90:204-224) ----
    if (spectrum) {
        DevBuf& bTmp = ctx->slot(8);
        DevBuf& bTot = ctx->slot(10);
        NRG_TRY(bTmp.ensure(sizeof(double) * 2 * nw));
        NRG_TRY(bTot.ensure(sizeof(double) * 4 * M.nMat));
        for (int N = startTrancation; N <= nIter; ++N) {
            const int idx = N - first;
            IterView V;
            V.S = &ctx->iter_sectors[idx]; V.kept = recs[idx].kept; V.d_V = slotV(idx).as<double>();
            V.d_Esec = slotE(idx).as<double>(); V.nb_kept = recs[idx].nb_kept;
            V.d_rdm = bRdm.as<double>(); V.rdm_off = recs[idx].rdm_off;
            const int nbo = recs[idx - 1].nb_kept;
            const double* dIMSprev = slotS(idx - 1).as<double>();
            if (N == nIter) {
                std::vector<int> gs;
                const Sectors& S = *V.S;
                for (int s = 0; s < S.nsub; ++s)
                    for (int p = 0; p < S.dim[s]; ++p)
                        if (recs[idx].Esec[S.start[s] + p] < 1.0e-8) gs.push_back(s);
                NRG_TRY(spike_t0_device(ctx, N, V, gs, nbo, dIMSprev, dPos, dNeg));
            } else {
                double* tPos = bTmp.as<double>();
                double* tNeg = tPos + nw;
                NRG_TRY(run_fill(ctx, tPos, (long long)(2 * nw), 0.0));
                NRG_TRY(spike_cfs_device(ctx, N, V, nbo, dIMSprev, bRdm.as<double>(), tPos, tNeg, bTot.as<double>()));
                NRG_TRY(run_add(ctx, dPos, tPos, (long long)(2 * nw)));
            }
        }
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[3], st));
    NRG_CUDA_TRY(cudaStreamSynchronize(st));
    NRG_TRY(check_device_status(ctx));

    if (out) {
        out->numberOfBin = nbin;
        out->startTrancation = startTrancation;
        if (out->binnedSpikePositive && out->binnedSpikeNegative && out->binCapacity >= (int64_t)(2 * nw) && spectrum) {
            for (int m = 0; m < M.nMat; ++m)
                for (int i = 0; i < nbin; ++i) {
                    const double e = std::pow(10.0, -15.0 + double(i) / 1000.0);
                    out->binnedSpikePositive[(size_t)m * nbin + i] = e;
                    out->binnedSpikeNegative[(size_t)m * nbin + i] = -e;
                }
            NRG_CUDA_TRY(cudaMemcpy(out->binnedSpikePositive + nw, dPos, sizeof(double) * nw, cudaMemcpyDeviceToHost));
            NRG_CUDA_TRY(cudaMemcpy(out->binnedSpikeNegative + nw, dNeg, sizeof(double) * nw, cudaMemcpyDeviceToHost));
        }
        if (out->finalEigenvalue) {
            const IterRec& RL = recs[last];
            for (int i = 0; i < out->finalCapacity && i < RL.nb_full; ++i) out->finalEigenvalue[i] = RL.Esec[i];
        }
        if (out->phaseSeconds) {
            float a = 0, b = 0, c = 0;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            cudaEventElapsedTime(&c, ev[2], ev[3]);
            out->phaseSeconds[0] = a * 1e-3;
            out->phaseSeconds[1] = b * 1e-3;
            out->phaseSeconds[2] = c * 1e-3;
            out->phaseSeconds[3] = (a + b + c) * 1e-3;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return NRG_OK;
}
