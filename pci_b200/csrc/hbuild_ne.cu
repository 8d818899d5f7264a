// One electron count of the FormH / FormJ kernels (compiled with -DPCI_NE=n
// for n = 1..8 so the template instantiations build in parallel).
#include "hbuild_impl.cuh"

#ifndef PCI_NE
#error "compile with -DPCI_NE=<electron count>"
#endif

#define PCI_CAT2(a, b) a##b
#define PCI_CAT(a, b) PCI_CAT2(a, b)

int PCI_CAT(hb_adjacency_ne, PCI_NE)(pci_gpu *h, DevSys S, const int32_t *d_ndc)
{
    return adjacency_impl<PCI_NE>(h, S, d_ndc);
}

int PCI_CAT(hb_rows_ne, PCI_NE)(pci_gpu *h, int kind, int value_prec, Csr &out, RowStatsOut *hs)
{
    RowStats r;
    int rc = kind == 0 ? rows_impl<PCI_NE, 0>(h, value_prec, out, &r) : rows_impl<PCI_NE, 1>(h, value_prec, out, &r);
    if (rc == PCI_OK) {
        hs->numzero = r.numzero;
        hs->pairs = r.pairs;
        hs->scanned = r.scanned;
        hs->hmin = (out.nnz > 0) ? key_to_double(r.hmin_key) : 0.0;
    }
    return rc;
}
