// C ABI of libpci_gpu.so: handle lifecycle, input validation and upload,
// CSR copy-out, and dispatch to the H-build, SpMM and Davidson units.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "pci_internal.h"

// ------------------------------------------------------------ helpers ---

int set_err(pci_gpu *h, int code, const std::string &msg)
{
    if (h) h->err = msg;
    return code;
}

int cuda_err(pci_gpu *h, cudaError_t e, const char *what)
{
    std::string m = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what;
    return set_err(h, e == cudaErrorMemoryAllocation ? PCI_E_OOM : PCI_E_CUDA, m);
}

void *dev_alloc(pci_gpu *h, size_t bytes, int *rc)
{
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess && h && spare_bytes(h) > 0) {
        // the buffers kept for reuse give way to any other allocation
        cudaGetLastError();
        spare_release(h);
        e = cudaMalloc(&p, bytes ? bytes : 16);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *rc = set_err(h, PCI_E_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        return nullptr;
    }
    *rc = PCI_OK;
    return p;
}

void dev_free(void *p)
{
    if (p) cudaFree(p);
}

int ensure_tmp(pci_gpu *h, size_t bytes)
{
    if (h->tmp_bytes >= bytes && h->d_tmp) return PCI_OK;
    cudaStreamSynchronize(h->st);
    dev_free(h->d_tmp);
    h->d_tmp = nullptr;
    h->tmp_bytes = 0;
    int rc = 0;
    h->d_tmp = dev_alloc(h, bytes, &rc);
    if (rc) return rc;
    h->tmp_bytes = bytes;
    return PCI_OK;
}

DevSys make_devsys(const pci_gpu *h)
{
    DevSys S;
    memset(&S, 0, sizeof(S));
    S.ne = h->ne; S.nst = h->nst; S.nsu = h->nsu; S.nso = h->nso; S.nx = h->nx; S.mj = h->mj; S.nc = h->nc;
    S.nlx = h->nlx; S.kbrt = h->kbrt; S.kdim = h->kdim; S.ntype = h->ntype;
    // per-tile term lists take the m-states of one orbital to precede those of
    // every later orbital (Nh non-decreasing) and carry no Breit term
    S.plans = (h->kbrt == 0 && std::is_sorted(h->h_nh.begin(), h->h_nh.end())) ? 1 : 0;
    S.nd = h->nd; S.gj = h->gj;
    S.occ = h->d_occ; S.conf_of = h->d_conf_of; S.conf_start = h->d_conf_start; S.conf_orb = h->d_conf_orb;
    S.adj_ptr = h->d_adj_ptr; S.adj = h->d_adj;
    S.ms_orb = h->d_ms_orb; S.ms_jz = h->d_ms_jz; S.ms_type = h->d_ms_type; S.msd = h->d_msd;
    S.orb_l = h->d_orb_l; S.orb_j = h->d_orb_j;
    S.h1 = h->d_h1; S.gaunt = h->d_gaunt; S.htab = h->d_htab; S.hw = h->hw;
    S.hmask = h->hcap ? h->hcap - 1 : 0;
    S.err = h->d_err;
    return S;
}

static int type_offset(int j2) { return ((j2 - 1) / 2) * ((j2 + 1) / 2); }

template <typename T>
static int upload(pci_gpu *h, T **dst, const std::vector<T> &src)
{
    int rc = 0;
    dev_free(*dst);
    *dst = (T *)dev_alloc(h, std::max<size_t>(src.size(), 1) * sizeof(T), &rc);
    if (rc) return rc;
    if (!src.empty()) PCI_CUDA(h, cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, h->st));
    return PCI_OK;
}

static void free_basis(pci_gpu *h)
{
    dev_free(h->d_occ); dev_free(h->d_conf_of); dev_free(h->d_conf_start); dev_free(h->d_conf_orb);
    dev_free(h->d_adj_ptr); dev_free(h->d_adj); dev_free(h->d_ms_orb); dev_free(h->d_ms_jz);
    dev_free(h->d_ms_type); dev_free(h->d_orb_l); dev_free(h->d_orb_j); dev_free(h->d_msd);
    dev_free(h->d_barr);
    dev_free(h->d_orb_n);
    h->d_orb_n = nullptr;
    dev_free(h->d_csf_C); dev_free(h->d_csf_start); dev_free(h->d_csf_coff);
    h->d_csf_C = nullptr; h->d_csf_start = nullptr; h->d_csf_coff = nullptr;
    h->h_csf_start.clear();
    h->ncsf = 0;
    dev_free(h->d_lsj_items);
    h->d_lsj_items = nullptr;
    h->lsj_nitems = -1;
    h->d_msd = nullptr;
    h->d_barr = nullptr;
    h->nint = 0;
    h->d_occ = nullptr; h->d_conf_of = nullptr; h->d_conf_start = nullptr; h->d_conf_orb = nullptr;
    h->d_adj_ptr = nullptr; h->d_adj = nullptr; h->d_ms_orb = nullptr; h->d_ms_jz = nullptr;
    h->d_ms_type = nullptr; h->d_orb_l = nullptr; h->d_orb_j = nullptr;
    h->have_basis = false;
}

// Gaunt table over (k, (j1,m1) type, (j2,m2) type) and the compact one-electron
// table need both the basis and the integrals; rebuilt whenever either changes.
static int build_tables(pci_gpu *h, const double *hint_lut, int nlx, int64_t nglut, const double *glut)
{
    int jmax2 = 1;
    for (int o = 0; o < h->nsu; o++) jmax2 = std::max(jmax2, h->h_orb_j[o]);
    h->kdim = jmax2 + 1;
    h->ntype = type_offset(jmax2 + 2);
    h->nlx = nlx;
    std::vector<double> g((size_t)h->kdim * h->ntype * h->ntype, 0.0);
    for (int k = 0; k < h->kdim; k++)
        for (int j1 = 1; j1 <= jmax2; j1 += 2)
            for (int m1 = -j1; m1 <= j1; m1 += 2)
                for (int j2 = 1; j2 <= jmax2; j2 += 2)
                    for (int m2 = -j2; m2 <= j2; m2 += 2) {
                        int t1 = type_offset(j1) + (m1 + j1) / 2, t2 = type_offset(j2) + (m2 + j2) / 2;
                        g[((size_t)k * h->ntype + t1) * h->ntype + t2] =
                            host_gaunt(nlx, glut, nglut, k, j1 * 0.5, m1 * 0.5, j2 * 0.5, m2 * 0.5);
                    }
    int rc = upload(h, &h->d_gaunt, g);
    if (rc) return rc;
    std::vector<double> h1((size_t)h->nsu * h->nsu, 0.0);
    for (int a = 0; a < h->nsu; a++)
        for (int b = 0; b < h->nsu; b++) {
            if (h->h_orb_k[a] != h->h_orb_k[b]) continue;
            int na = std::min(a, b) + 1, nb = std::max(a, b) + 1;  // 1-based, na <= nb
            int64_t ind = (int64_t)h->nx * (na - h->nso - 1) + (nb - h->nso);
            if (ind >= 1 && ind <= (int64_t)h->nx * h->nx) h1[(size_t)a * h->nsu + b] = hint_lut[ind - 1];
        }
    return upload(h, &h->d_h1, h1);
}

// ---------------------------------------------------------------- ABI ---

extern "C" {

int pci_gpu_create(int32_t device, pci_gpu_t **out)
{
    if (!out) return PCI_E_INPUT;
    *out = nullptr;
    pci_gpu *h = new pci_gpu();
    h->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        int rc = cuda_err(h, e, "cudaSetDevice");
        *out = h;  // keep the handle so the caller can read the message
        return rc;
    }
    e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { *out = h; return cuda_err(h, e, "cudaStreamCreate"); }
    int rc = 0;
    h->d_err = (unsigned int *)dev_alloc(h, 16, &rc);
    if (rc) { *out = h; return rc; }
    if (const char *m = getenv("PCI_SPMM")) {
        if (!strcmp(m, "full")) h->spmm_mode = 1;
        else if (!strcmp(m, "lower")) h->spmm_mode = 2;
    }
    cudaMemset(h->d_err, 0, 16);
    *out = h;
    return PCI_OK;
}

// Jt(1:Njd), the sorted 2J values of the terms the configurations hold, as
// Dinit finds them (src/determinants.f90:227-325): per configuration with
// determinants at 2M = Mj, the number of its determinants at each
// 2M = Mj + 2(im-1) >= Mj; terms are peeled off from the largest im down.
// The counts come from the m-value distribution of each orbital's
// occupation (subsets of its 2j+1 m values) convolved over the orbitals,
// instead of enumerating the determinants.
static std::vector<int32_t> compute_jterms(int Ne, int Nc, const int32_t *Ndc, const std::vector<uint16_t> &conf_orb,
                                           const int32_t *Jj, int Nsu, int Mj)
{
    std::vector<int32_t> jt;
    int jmax = 1;
    for (int o = 0; o < Nsu; o++) jmax = std::max(jmax, (int)Jj[o]);
    const int OFF = Ne * jmax;  // |2M| <= Ne * max(2j)
    // The terms of a configuration depend only on its (2j, occupation) groups:
    // configurations with the same groups share one computation.
    std::map<std::vector<int>, std::vector<int32_t>> memo;
    for (int c = 0; c < Nc; c++) {
        if (Ndc[c] == 0) continue;
        std::vector<int> orbs(conf_orb.begin() + (size_t)c * Ne, conf_orb.begin() + (size_t)(c + 1) * Ne);
        std::sort(orbs.begin(), orbs.end());
        std::vector<int> key;   // (2j, q) of each orbital group, sorted
        for (size_t i = 0; i < orbs.size();) {
            size_t j = i;
            while (j < orbs.size() && orbs[j] == orbs[i]) j++;
            key.push_back(Jj[orbs[i]] * 16 + (int)(j - i));
            i = j;
        }
        std::sort(key.begin(), key.end());
        auto it = memo.find(key);
        if (it == memo.end()) {
            std::vector<int64_t> dist(2 * OFF + 1, 0);
            dist[OFF] = 1;
            for (int kq : key) {
                const int q = kq % 16, j2 = kq / 16;
                // ways[k][s]: k of the m values -j2, -j2+2, ..., j2 chosen with 2M sum s
                std::vector<std::vector<int64_t>> ways(q + 1, std::vector<int64_t>(2 * OFF + 1, 0));
                ways[0][OFF] = 1;
                for (int m = -j2; m <= j2; m += 2)
                    for (int k = q; k >= 1; k--)
                        for (int sidx = 0; sidx <= 2 * OFF; sidx++)
                            if (ways[k - 1][sidx] && sidx + m >= 0 && sidx + m <= 2 * OFF) ways[k][sidx + m] += ways[k - 1][sidx];
                std::vector<int64_t> nd2(2 * OFF + 1, 0);
                for (int a = 0; a <= 2 * OFF; a++)
                    if (dist[a])
                        for (int b = 0; b <= 2 * OFF; b++)
                            if (ways[q][b] && a + b - OFF >= 0 && a + b - OFF <= 2 * OFF) nd2[a + b - OFF] += dist[a] * ways[q][b];
                dist.swap(nd2);
            }
            std::vector<int32_t> mts;
            if (Mj + OFF >= 0 && Mj + OFF <= 2 * OFF && dist[Mj + OFF] != 0) {
                std::vector<int64_t> nmj(1, 0);   // nmj[im], im >= 1
                for (int m2 = Mj; m2 + OFF <= 2 * OFF; m2 += 2) nmj.push_back(dist[m2 + OFF]);
                int imax = (int)nmj.size() - 1;
                while (imax > 1 && nmj[imax] == 0) imax--;
                for (int im = imax; im >= 1; im--) {
                    const int64_t n = nmj[im];
                    if (n != 0) {
                        for (int k = 1; k <= im; k++) nmj[k] -= n;
                        mts.push_back((im - 1) * 2 + Mj);
                    }
                }
            }
            it = memo.emplace(key, std::move(mts)).first;
        }
        for (int32_t mt : it->second)
            if (std::find(jt.begin(), jt.end(), mt) == jt.end()) jt.push_back(mt);
    }
    std::sort(jt.begin(), jt.end());
    return jt;
}

int pci_gpu_jterms(pci_gpu_t *h, int32_t *out, int32_t cap)
{
    if (!h || !h->have_basis) return -1;
    const int32_t n = (int32_t)h->h_jterms.size();
    for (int32_t i = 0; i < n && out && i < cap; i++) out[i] = h->h_jterms[(size_t)i];
    return n;
}

int pci_gpu_set_basis(pci_gpu_t *h, int32_t Ne, int64_t Nd, int32_t Nst, int32_t Nsu, int32_t Nso, int32_t Nx,
                      int32_t Mj, const int32_t *Iarr, const int32_t *Nh, const int32_t *Jz, const int32_t *Nn,
                      const int32_t *Kk, const int32_t *Ll, const int32_t *Jj, int32_t Nc, const int32_t *Ndc,
                      double Gj)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (Ne < 1 || Ne > PCI_NE_MAX) return set_err(h, PCI_E_INPUT, "Ne must be 1..8");
    if (Nd < 1 || Nd >= (1LL << 31)) return set_err(h, PCI_E_INPUT, "Nd out of range");
    if (Nst < 1 || Nst > 65000) return set_err(h, PCI_E_INPUT, "Nst out of range");
    if (Nsu < 1 || Nc < 1 || Nx < 1 || Nso < 0) return set_err(h, PCI_E_INPUT, "bad Nsu/Nc/Nx/Nso");
    if (!Iarr || !Nh || !Jz || !Kk || !Ll || !Jj || !Ndc) return set_err(h, PCI_E_INPUT, "null array");
    int64_t sum = 0;
    for (int c = 0; c < Nc; c++) {
        if (Ndc[c] < 0) return set_err(h, PCI_E_INPUT, "negative Ndc");
        sum += Ndc[c];
    }
    if (sum != Nd) return set_err(h, PCI_E_INPUT, "sum(Ndc) /= Nd");
    for (int i = 0; i < Nst; i++) {
        if (Nh[i] < 1 || Nh[i] > Nsu) return set_err(h, PCI_E_INPUT, "Nh outside 1..Nsu");
        int j2 = Jj[Nh[i] - 1];
        if (j2 < 1 || j2 > 63 || (j2 & 1) == 0 || Jz[i] < -j2 || Jz[i] > j2 || ((Jz[i] + j2) & 1))
            return set_err(h, PCI_E_INPUT, "Jz inconsistent with Jj");
    }
    if (Nsu - Nso > Nx) return set_err(h, PCI_E_INPUT, "Nsu - Nso exceeds Nx");
    free_basis(h);
    csr_retire(h, h->H); csr_free(h->J); csr_free(h->Hfull);
    h->ne = Ne; h->nd = Nd; h->nst = Nst; h->nsu = Nsu; h->nso = Nso; h->nx = Nx; h->mj = Mj; h->nc = Nc; h->gj = Gj;
    h->h_ndc.assign(Ndc, Ndc + Nc);
    h->h_orb_j.assign(Jj, Jj + Nsu);
    h->h_orb_l.assign(Ll, Ll + Nsu);
    h->h_orb_k.assign(Kk, Kk + Nsu);
    if (Nn) h->h_orb_n.assign(Nn, Nn + Nsu);
    else h->h_orb_n.clear();
    h->h_nh.assign(Nh, Nh + Nst);
    h->h_jz.assign(Jz, Jz + Nst);
    // determinants: 0-based uint16, validated sorted and configuration-consistent
    std::vector<uint16_t> occ((size_t)Nd * Ne);
    std::vector<int32_t> conf_of(Nd);
    std::vector<int64_t> conf_start(Nc + 1);
    std::vector<uint16_t> conf_orb((size_t)Nc * Ne, 0);
    conf_start[0] = 0;
    for (int c = 0; c < Nc; c++) conf_start[c + 1] = conf_start[c] + Ndc[c];
    for (int c = 0; c < Nc; c++) {
        for (int64_t n = conf_start[c]; n < conf_start[c + 1]; n++) {
            conf_of[n] = c;
            for (int e = 0; e < Ne; e++) {
                int32_t m = Iarr[n * Ne + e];
                if (m < 1 || m > Nst) return set_err(h, PCI_E_INPUT, "Iarr entry outside 1..Nst at det " + std::to_string(n + 1));
                if (e > 0 && m <= Iarr[n * Ne + e - 1])
                    return set_err(h, PCI_E_INPUT, "RSPQ: determinant not sorted ascending at det " + std::to_string(n + 1));
                occ[n * Ne + e] = (uint16_t)(m - 1);
                uint16_t o = (uint16_t)(Nh[m - 1] - 1);
                if (n == conf_start[c]) conf_orb[(size_t)c * Ne + e] = o;
                else if (conf_orb[(size_t)c * Ne + e] != o)
                    return set_err(h, PCI_E_INPUT, "determinant " + std::to_string(n + 1) + " does not belong to its configuration block");
            }
        }
    }
    h->h_jterms = compute_jterms(Ne, Nc, Ndc, conf_orb, Jj, Nsu, Mj);
    std::vector<int16_t> ms_orb(Nst);
    std::vector<int8_t> ms_jz(Nst), orb_l(Nsu), orb_j(Nsu);
    std::vector<uint8_t> ms_type(Nst);
    std::vector<uint32_t> msd(Nst);
    if (Nsu > 1024) return set_err(h, PCI_E_INPUT, "Nsu above 1024");
    for (int i = 0; i < Nst; i++) {
        ms_orb[i] = (int16_t)(Nh[i] - 1);
        ms_jz[i] = (int8_t)Jz[i];
        int j2 = Jj[Nh[i] - 1];
        int l = Ll[Nh[i] - 1];
        int type = type_offset(j2) + (Jz[i] + j2) / 2;
        if (j2 > 31 || l > 15 || type > 63) return set_err(h, PCI_E_INPUT, "orbital j or l out of range (2j <= 31, l <= 15)");
        ms_type[i] = (uint8_t)type;
        msd[i] = (uint32_t)(Nh[i] - 1) | ((uint32_t)type << 10) | ((uint32_t)(Jz[i] + 128) << 16) |
                 ((uint32_t)l << 24) | ((uint32_t)((j2 - 1) / 2) << 28);
    }
    for (int o = 0; o < Nsu; o++) { orb_l[o] = (int8_t)Ll[o]; orb_j[o] = (int8_t)Jj[o]; }
    int rc;
    if ((rc = upload(h, &h->d_occ, occ))) return rc;
    if ((rc = upload(h, &h->d_conf_of, conf_of))) return rc;
    if ((rc = upload(h, &h->d_conf_start, conf_start))) return rc;
    if ((rc = upload(h, &h->d_conf_orb, conf_orb))) return rc;
    if ((rc = upload(h, &h->d_ms_orb, ms_orb))) return rc;
    if ((rc = upload(h, &h->d_ms_jz, ms_jz))) return rc;
    if ((rc = upload(h, &h->d_ms_type, ms_type))) return rc;
    if ((rc = upload(h, &h->d_msd, msd))) return rc;
    if ((rc = upload(h, &h->d_orb_l, orb_l))) return rc;
    if ((rc = upload(h, &h->d_orb_j, orb_j))) return rc;
    if (Nn) {
        std::vector<int8_t> orb_n(Nsu);
        for (int o = 0; o < Nsu; o++) {
            if (Nn[o] < 1 || Nn[o] > 127) return set_err(h, PCI_E_INPUT, "Nn outside 1..127");
            orb_n[o] = (int8_t)Nn[o];
        }
        if ((rc = upload(h, &h->d_orb_n, orb_n))) return rc;
    }
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    h->have_basis = true;
    h->have_ints = false;  // tables depend on the basis; integrals must be set again
    return PCI_OK;
}

int pci_gpu_set_integrals(pci_gpu_t *h, const double *HintLUT, int32_t Nlx, int64_t nGauntLUT, const double *GauntLUT,
                          int64_t Ngint, int32_t kbrt, int32_t r2_is_f64, const void *Rint2, const int32_t *Iint2,
                          const int32_t *Iint3)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "set_integrals before set_basis");
    if (!HintLUT || !GauntLUT || !Rint2 || !Iint2 || !Iint3) return set_err(h, PCI_E_INPUT, "null array");
    if (Nlx < 0 || nGauntLUT < 1) return set_err(h, PCI_E_INPUT, "bad Gaunt table");
    int rc;
    if ((rc = build_tables(h, HintLUT, Nlx, nGauntLUT, GauntLUT))) return rc;
    if ((rc = hb_build_hash(h, Ngint, kbrt, r2_is_f64, Rint2, Iint2, Iint3))) return rc;
    csr_retire(h, h->H); csr_free(h->J); csr_free(h->Hfull);
    h->have_ints = true;
    return PCI_OK;
}

int pci_gpu_form_h(pci_gpu_t *h, int32_t value_prec, int64_t *NumH, int64_t *numzero, double *Hmin)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    return hb_form_h(h, value_prec, NumH, numzero, Hmin);
}

int pci_gpu_form_h_pt(pci_gpu_t *h, int64_t nd1, int64_t nd0, int32_t value_prec, int64_t *NumH)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "form_h_pt before set_basis/set_integrals");
    return hb_form_h_pt(h, nd1, nd0, nd1, h->nd, value_prec, NumH);
}

int pci_gpu_form_h_pt_rows(pci_gpu_t *h, int64_t nd1, int64_t nd0, int64_t row_lo, int64_t row_hi,
                           int32_t value_prec, int64_t *NumH)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    return hb_form_h_pt(h, nd1, nd0, row_lo, row_hi, value_prec, NumH);
}

int pci_gpu_form_j(pci_gpu_t *h, int64_t *NumJ)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    return hb_form_j(h, NumJ);
}

int pci_gpu_csr_info(pci_gpu_t *h, int32_t which, int64_t *nrows, int64_t *nnz)
{
    if (!h) return PCI_E_INPUT;
    const Csr &c = which == PCI_MAT_J2 ? h->J : h->H;
    if (!c.rowptr) return set_err(h, PCI_E_STATE, "matrix not formed");
    if (nrows) *nrows = c.nrows;
    if (nnz) *nnz = c.nnz;
    return PCI_OK;
}

int pci_gpu_get_csr(pci_gpu_t *h, int32_t which, int64_t *rowptr, int32_t *col, double *val)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    const Csr &c = which == PCI_MAT_J2 ? h->J : h->H;
    if (!c.rowptr) return set_err(h, PCI_E_STATE, "matrix not formed");
    if (rowptr) PCI_CUDA(h, cudaMemcpy(rowptr, c.rowptr, (c.nrows + 1) * 8, cudaMemcpyDeviceToHost));
    if (col) {
        PCI_CUDA(h, cudaMemcpy(col, c.col, c.nnz * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < c.nnz; i++) col[i] += 1;  // Fortran 1-based columns
    }
    if (val) {
        if (c.val_f32) {
            std::vector<float> tmp(c.nnz);
            PCI_CUDA(h, cudaMemcpy(tmp.data(), c.val, c.nnz * 4, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < c.nnz; i++) val[i] = tmp[i];
        } else {
            PCI_CUDA(h, cudaMemcpy(val, c.val, c.nnz * 8, cudaMemcpyDeviceToHost));
        }
    }
    return PCI_OK;
}

int pci_gpu_get_csr_rows(pci_gpu_t *h, int32_t which, int64_t row_lo, int64_t row_hi, int64_t *rowptr, int32_t *col,
                         double *val)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    const Csr &c = which == PCI_MAT_J2 ? h->J : h->H;
    if (!c.rowptr) return set_err(h, PCI_E_STATE, "matrix not formed");
    if (!rowptr || row_lo < 1 || row_hi < row_lo || row_hi > c.nrows)
        return set_err(h, PCI_E_INPUT, "get_csr_rows: need 1 <= row_lo <= row_hi <= Nd and rowptr");
    const int64_t n = row_hi - row_lo + 1;
    PCI_CUDA(h, cudaMemcpy(rowptr, c.rowptr + (row_lo - 1), (n + 1) * 8, cudaMemcpyDeviceToHost));
    const int64_t base = rowptr[0], cnt = rowptr[n] - base;
    for (int64_t i = 0; i <= n; i++) rowptr[i] -= base;
    if (col && cnt) {
        PCI_CUDA(h, cudaMemcpy(col, c.col + base, cnt * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < cnt; i++) col[i] += 1;   // Fortran 1-based columns
    }
    if (val && cnt) {
        if (c.val_f32) {
            std::vector<float> tmp(cnt);
            PCI_CUDA(h, cudaMemcpy(tmp.data(), (const float *)c.val + base, cnt * 4, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < cnt; i++) val[i] = tmp[i];
        } else {
            PCI_CUDA(h, cudaMemcpy(val, (const double *)c.val + base, cnt * 8, cudaMemcpyDeviceToHost));
        }
    }
    return PCI_OK;
}

int pci_gpu_set_csr(pci_gpu_t *h, int32_t which, int64_t Nd, int64_t nnz, const int64_t *rowptr, const int32_t *col,
                    const double *val, double Hmin)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!rowptr || !col || !val || Nd < 1 || nnz < 0) return set_err(h, PCI_E_INPUT, "bad CSR");
    if (h->have_basis && Nd != h->nd) return set_err(h, PCI_E_INPUT, "CSR rows differ from Nd");
    if (rowptr[0] != 0 || rowptr[Nd] != nnz) return set_err(h, PCI_E_INPUT, "rowptr inconsistent with nnz");
    Csr &c = which == PCI_MAT_J2 ? h->J : h->H;
    csr_free(c);
    if (which != PCI_MAT_J2) {
        csr_free(h->Hfull);
        h->h_from_tiles = false;
        h->h_pt_nd1 = -1;
    }
    int rc = 0;
    c.nrows = Nd;
    c.nnz = nnz;
    c.val_f32 = 0;
    c.rowptr = (int64_t *)dev_alloc(h, (Nd + 1) * 8, &rc);
    if (rc) return rc;
    c.col = (int32_t *)dev_alloc(h, std::max<int64_t>(nnz, 1) * 4, &rc);
    if (rc) return rc;
    c.val = dev_alloc(h, std::max<int64_t>(nnz, 1) * 8, &rc);
    if (rc) return rc;
    std::vector<int32_t> c0(nnz);
    for (int64_t i = 0; i < nnz; i++) {
        if (col[i] < 1 || col[i] > Nd) return set_err(h, PCI_E_INPUT, "column outside 1..Nd");
        c0[i] = col[i] - 1;
    }
    PCI_CUDA(h, cudaMemcpy(c.rowptr, rowptr, (Nd + 1) * 8, cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemcpy(c.col, c0.data(), nnz * 4, cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemcpy(c.val, val, nnz * 8, cudaMemcpyHostToDevice));
    if (which != PCI_MAT_J2) {
        h->hmin = Hmin;
        h->numh = nnz;
        if (!h->have_basis) h->nd = Nd;
    }
    return PCI_OK;
}

int pci_gpu_davidson(pci_gpu_t *h, const pci_dvd_params *p, const double *X0, double *Tk, double *Tj,
                     int32_t *Iconverge, double *X, int32_t *iters, double *resid)
{
    if (!h || !p) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (h->H.rowptr && h->H.nrows != h->nd)
        return set_err(h, PCI_E_STATE, "davidson: the resident matrix is the CSF one; solve it with the batched solver");
    if (h->H.rowptr && h->h_pt_nd1 >= 0)
        return set_err(h, PCI_E_STATE, "davidson: the resident matrix is conf_pt's PT block (pci_gpu_form_h_pt)");
    return dv_run(h, p, X0, Tk, Tj, Iconverge, X, iters, resid);
}

int pci_gpu_davidson_harvest(pci_gpu_t *h, const pci_dvd_params *p, const double *Xref, float *feat, float *target,
                             int64_t cap, int64_t *count, double *Tk, int32_t *Iconverge, int32_t *iters)
{
    if (!h || !p || !count) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (p->mode != PCI_DVD_FP64) return set_err(h, PCI_E_INPUT, "harvest runs the FP64 form");
    if (h->H.rowptr && (h->H.nrows != h->nd || h->h_pt_nd1 >= 0))
        return set_err(h, PCI_E_STATE, "harvest needs the determinant H of pci_gpu_form_h");
    DvdHarvest hv;
    hv.feat = feat;
    hv.target = target;
    hv.cap = cap;
    hv.xref = Xref;
    std::vector<double> tj(p->Nlv);
    int rc = dv_run(h, p, nullptr, Tk, tj.data(), Iconverge, nullptr, iters, nullptr, &hv);
    *count = hv.count;
    return rc;
}

int pci_gpu_set_correction_model(pci_gpu_t *h, pci_mlp_t *m)
{
    if (!h) return PCI_E_INPUT;
    h->corr_model = m;
    return PCI_OK;
}

int pci_gpu_j_av(pci_gpu_t *h, const double *X, int32_t nv, int64_t nlim, double *Tj)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!X || !Tj) return set_err(h, PCI_E_INPUT, "null array");
    if (!h->J.rowptr) return set_err(h, PCI_E_STATE, "J_av before form_j");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "J_av: nv must be 1..64");
    const int64_t nd = h->J.nrows;
    int rc = 0;
    double *d = (double *)dev_alloc(h, (size_t)nd * nv * 8, &rc);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(d, X, (size_t)nd * nv * 8, cudaMemcpyHostToDevice, h->st);
    if (e != cudaSuccess) { dev_free(d); return cuda_err(h, e, "cudaMemcpyAsync"); }
    rc = sp_jav_strided(h, d, 1, nd, nv, nlim, Tj);
    cudaStreamSynchronize(h->st);
    dev_free(d);
    return rc;
}

int32_t pci_gpu_stats(pci_gpu_t *h, double *out, int32_t n)
{
    if (!h || !out) return 0;
    double v[15] = {h->st_formh, h->st_formh_count, h->st_formh_fill, h->st_formj,
                    h->st_dvd, h->st_spmm, h->st_spmm_calls, h->st_init,
                    h->st_adj, h->st_pairs, h->st_scanned, h->st_launches,
                    h->st_formh_compact, h->st_formh_padded, h->st_formh_slots};
    int32_t m = std::min<int32_t>(n, 15);
    for (int i = 0; i < m; i++) out[i] = v[i];
    return m;
}

const char *pci_gpu_last_error(pci_gpu_t *h)
{
    return h ? h->err.c_str() : "null handle";
}

// ----------------------------------------------------- bit-string path ---

// FormBarr (src/determinants.f90:839-864): bit m-1 of determinant n's bit
// string is set for each occupied m-state m (1-based): word (m-1)/32, bit
// (m-1) mod 32; Barr is nint x Nd, column-major.
__global__ void k_form_barr(const uint16_t *occ, int ne, int64_t nd, int nint, int32_t *barr)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        int32_t *b = barr + n * nint;
        for (int w = 0; w < nint; w++) b[w] = 0;
        for (int e = 0; e < ne; e++) {
            const int m = occ[n * ne + e];   // 0-based m-state = (1-based) - 1
            b[m >> 5] |= (int32_t)(1u << (m & 31));
        }
    }
}

// compare_bit_dets + get_det_indexes (src/determinants.f90:933-1034) for
// one pair of bit strings, step for step: the difference count from the
// popcount of the XOR (3 when it reaches 6 differing bits), then for 1 or 2
// differences the differing positions (1-based) of each determinant and the
// phase from the positions less the zero bits seen after the first occupied
// one.  The early exit leaves only the bit loop of the current word, as the
// reference's `exit` does, so later words still add to the zero-bit count.
__device__ void d_bit_compare(const int32_t *b1, const int32_t *b2, int nint, int &ndiffs, int &is, int *d1, int *d2)
{
    int nf = 0;
    ndiffs = -1;
    for (int w = 0; w < nint; w++) {
        if (b1[w] != 0 || b2[w] != 0) {
            nf += __popc((uint32_t)(b1[w] ^ b2[w]));
            if (nf >= 6) {
                ndiffs = 3;
                break;
            }
        }
    }
    if (ndiffs < 0) ndiffs = (nf + 1) / 2;
    d1[0] = d1[1] = d1[2] = 0;
    d2[0] = d2[1] = d2[2] = 0;
    is = 1;
    if (ndiffs > 2 || ndiffs == 0) return;
    int i1 = 1, j1 = 1, nzb = 0, first = 0, l1[2] = {0, 0}, l2[2] = {0, 0};
    for (int w = 0; w < nint; w++) {
        const uint32_t x1 = (uint32_t)b1[w], x2 = (uint32_t)b2[w];
        if (x1 == 0 && x2 == 0) continue;
        for (int bit = 0; bit < 32; bit++) {
            const int bt1 = (x1 >> bit) & 1, bt2 = (x2 >> bit) & 1;
            if (bt1 || bt2) first = 1;
            if (!bt1 && !bt2) {
                if (first) nzb++;
            } else if (bt1 != bt2) {
                const int pos = 32 * w + bit + 1;
                if (bt1) {
                    i1++;
                    if (i1 <= 3) { d1[i1 - 1] = pos; l1[i1 - 2] = pos - nzb; }
                }
                if (bt2) {
                    j1++;
                    if (j1 <= 3) { d2[j1 - 1] = pos; l2[j1 - 2] = pos - nzb; }
                }
                if ((ndiffs == 1 && i1 == 2 && j1 == 2) || (ndiffs == 2 && i1 == 3 && j1 == 3)) break;
            }
        }
    }
    if (ndiffs == 1) {
        if (nzb > 0 && abs(l2[0] - l1[0] - 1) % 2 == 1) is = -is;
    } else {
        if (abs(l2[0] - l1[0] - nzb % 2) % 2 == 1) is = -is;
        if (abs(l2[1] - l1[1] - nzb % 2) % 2 == 1) is = -is;
        int t = d2[1]; d2[1] = d2[2]; d2[2] = t;
        t = d1[1]; d1[1] = d1[2]; d1[2] = t;
    }
}

__global__ void k_bit_compare(const int32_t *barr, int nint, int64_t nd, const int64_t *pairs, int64_t n, int32_t *ndiffs,
                              int32_t *is, int32_t *idx1, int32_t *idx2, unsigned *err)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = pairs[2 * t] - 1, b = pairs[2 * t + 1] - 1;
        if (a < 0 || a >= nd || b < 0 || b >= nd) {
            atomicOr(err, DERR_BAD_INDEX);
            continue;
        }
        int nf, s, d1[3], d2[3];
        d_bit_compare(barr + a * nint, barr + b * nint, nint, nf, s, d1, d2);
        ndiffs[t] = nf;
        is[t] = s;
        for (int q = 0; q < 3; q++) {
            idx1[3 * t + q] = d1[q];
            idx2[3 * t + q] = d2[q];
        }
    }
}

int pci_gpu_form_barr(pci_gpu_t *h, int32_t *nint_out, int32_t *barr)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "form_barr before set_basis");
    const int nint = (h->nst + 31) / 32;
    if (!h->d_barr) {
        int rc = 0;
        h->d_barr = (int32_t *)dev_alloc(h, (size_t)nint * std::max<int64_t>(h->nd, 1) * 4, &rc);
        if (rc) return rc;
        h->nint = nint;
        k_form_barr<<<148 * 4, 256, 0, h->st>>>(h->d_occ, h->ne, h->nd, nint, h->d_barr);
        PCI_CUDA(h, cudaGetLastError());
    }
    if (nint_out) *nint_out = nint;
    if (barr) PCI_CUDA(h, cudaMemcpyAsync(barr, h->d_barr, (size_t)nint * h->nd * 4, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    return PCI_OK;
}

int pci_gpu_bit_compare(pci_gpu_t *h, int64_t n, const int64_t *pairs, int32_t *ndiffs, int32_t *is, int32_t *idx1,
                        int32_t *idx2)
{
    if (!h || n < 0 || (n && (!pairs || !ndiffs || !is || !idx1 || !idx2))) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!h->d_barr) return set_err(h, PCI_E_STATE, "bit_compare before form_barr");
    if (n == 0) return PCI_OK;
    int rc = 0;
    char *buf = (char *)dev_alloc(h, (size_t)n * (16 + 4 * 8), &rc);
    if (rc) return rc;
    int64_t *dp = (int64_t *)buf;
    int32_t *dn = (int32_t *)(buf + n * 16), *ds = dn + n, *d1 = ds + n, *d2 = d1 + 3 * n;
    PCI_CUDA(h, cudaMemsetAsync(h->d_err, 0, 4, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(dp, pairs, (size_t)n * 16, cudaMemcpyHostToDevice, h->st));
    k_bit_compare<<<148 * 4, 256, 0, h->st>>>(h->d_barr, h->nint, h->nd, dp, n, dn, ds, d1, d2, h->d_err);
    unsigned e = 0;
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(ndiffs, dn, (size_t)n * 4, cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(is, ds, (size_t)n * 4, cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(idx1, d1, (size_t)n * 12, cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(idx2, d2, (size_t)n * 12, cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&e, h->d_err, 4, cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
    dev_free(buf);
    if (ce != cudaSuccess) return cuda_err(h, ce, "bit_compare");
    if (e) return set_err(h, PCI_E_INPUT, "bit_compare: determinant index out of 1..Nd");
    return PCI_OK;
}

void pci_gpu_destroy(pci_gpu_t *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    free_basis(h);
    csr_free(h->H); csr_free(h->J); csr_free(h->Hfull);
    spare_release(h);
    dev_free(h->d_h1); dev_free(h->d_gaunt); dev_free(h->d_htab);
    dev_free(h->d_err); dev_free(h->d_tmp);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

}  // extern "C"
