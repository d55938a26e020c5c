// ref_dump.cc -- drives the reference's own host loaders and table
// derivation (gpudocksm-rem-1.2/src/load.C, data.C, util.C, compiled from the
// reference sources by oracle/Makefile.ref) the way dock.C:14-90 does, and
// dumps the kernel-ready tables so that the oracle can be pinned to the
// reference's own inputs (test infrastructure only).
//
//   ref_dump <pdb> <sdf> <lhm.ff> <params.ff> <weights> <nor_a> <nor_b>
//            <ligand_id> <out.bin>
//
// Output: a sequence of records  name\0 | type char | u64 count | payload.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "dock.h"
#include "load.h"
#include "util.h"

static FILE *g_out;

static void put(const char *name, char type, const void *data, uint64_t n, size_t elem) {
  fwrite(name, 1, strlen(name) + 1, g_out);
  fwrite(&type, 1, 1, g_out);
  fwrite(&n, sizeof(n), 1, g_out);
  fwrite(data, elem, n, g_out);
}

int main(int argc, char **argv) {
  if (argc != 10) {
    fprintf(stderr, "usage: %s pdb sdf lhm params weights nor_a nor_b ligand_id out\n", argv[0]);
    return 2;
  }
  InputFiles *in = new InputFiles[1];
  in->prt_file.path = argv[1];
  in->lig_file.path = argv[2];
  in->lig_file.molid = "MOLID";
  in->lhm_file.path = argv[3];
  in->enepara_file.path = argv[4];
  in->weight_file.path = argv[5];
  in->norpara_file.path_a = argv[6];
  in->norpara_file.path_b = argv[7];
  in->lhm_file.ligand_id = argv[8];

  Ligand0 *lig0 = new Ligand0[MAXEN2];
  Protein0 *prt0 = new Protein0[MAXEN1];
  Psp0 *psp0 = new Psp0;
  memset(psp0, 0, sizeof(Psp0));
  Kde0 *kde0 = new Kde0;
  memset(kde0, 0, sizeof(Kde0));
  Mcs0 *mcs0 = new Mcs0[MAXPOS];
  EnePara0 *ep0 = new EnePara0;
  memset(ep0, 0, sizeof(EnePara0));

  loadLigand(&in->lig_file, lig0);
  loadProtein(&in->prt_file, prt0);
  loadLHM(&in->lhm_file, psp0, kde0, mcs0);
  loadEnePara(&in->enepara_file, ep0);
  loadWeight(&in->weight_file, ep0);
  loadNorPara(&in->norpara_file, ep0);

  ComplexSize cs;
  cs.n_prt = in->prt_file.conf_total;
  cs.n_tmp = 1;
  cs.n_lig = in->lig_file.conf_total;
  cs.n_rep = cs.n_lig * cs.n_prt * cs.n_tmp;
  cs.lna = in->lig_file.lna;
  cs.pnp = in->prt_file.pnp;
  cs.pnk = kde0->pnk;
  cs.pos = in->lhm_file.pos;

  Ligand *lig = new Ligand[cs.n_lig];
  Protein *prt = new Protein[cs.n_prt];
  Psp *psp = new Psp;
  Kde *kde = new Kde;
  Mcs *mcs = new Mcs[cs.pos > 0 ? cs.pos : 1];
  EnePara *ep = new EnePara;
  OptimizeLigand(lig0, lig, cs);
  OptimizeProtein(prt0, prt, ep0, lig0, cs);
  OptimizePsp(psp0, psp, lig, prt);
  OptimizeKde(kde0, kde);
  OptimizeMcs(mcs0, mcs, cs);
  OptimizeEnepara(ep0, ep);
  InitLigCoord(lig, cs);

  g_out = fopen(argv[9], "wb");
  if (!g_out) return 3;
  int sizes[8] = {cs.n_lig, cs.n_prt, cs.lna, cs.pnp, cs.pnk, cs.pos, 0, 0};
  put("sizes", 'i', sizes, 8, 4);
  put("enepara_raw", 'b', ep0, sizeof(EnePara0), 1);
  put("enepara", 'b', ep, sizeof(EnePara), 1);
  for (int l = 0; l < cs.n_lig; ++l) {
    put("lig_x", 'f', lig[l].coord_orig.x, cs.lna, 4);
    put("lig_y", 'f', lig[l].coord_orig.y, cs.lna, 4);
    put("lig_z", 'f', lig[l].coord_orig.z, cs.lna, 4);
    put("lig_new_x", 'f', lig[l].coord_new.x, cs.lna, 4);
    put("lig_new_y", 'f', lig[l].coord_new.y, cs.lna, 4);
    put("lig_new_z", 'f', lig[l].coord_new.z, cs.lna, 4);
  }
  put("lig_center", 'f', lig[0].coord_orig.center, 3, 4);
  put("lig_t", 'i', lig[0].t, cs.lna, 4);
  put("lig_c", 'f', lig[0].c, cs.lna, 4);
  put("lig_n", 'i', lig[0].n, cs.lna, 4);
  for (int p = 0; p < cs.n_prt; ++p) {
    put("prt_x", 'f', prt[p].x, cs.pnp, 4);
    put("prt_y", 'f', prt[p].y, cs.pnp, 4);
    put("prt_z", 'f', prt[p].z, cs.pnp, 4);
  }
  put("prt_t", 'i', prt[0].t, cs.pnp, 4);
  put("prt_c", 'i', prt[0].c, cs.pnp, 4);
  put("prt_ele", 'f', prt[0].ele, cs.pnp, 4);
  put("prt_seq3r", 'i', prt[0].seq3r, cs.pnp, 4);
  put("prt_hpcflag", 'i', prt[0].c0_and_d12_or_c2, cs.pnp, 4);
  put("prt_hpp", 'f', prt[0].hpp, cs.pnp, 4);
  put("pocket_center", 'f', prt[0].pocket_center, 3, 4);
  int maxseq = 0;
  for (int p = 0; p < cs.pnp; ++p) maxseq = prt[0].seq3r[p] > maxseq ? prt[0].seq3r[p] : maxseq;
  const int ncol = maxseq + 1;
  for (int t = 0; t < MAXTP2; ++t) put("psp_row", 'f', psp->psp[t], ncol, 4);
  put("kde_x", 'f', kde->x, cs.pnk, 4);
  put("kde_y", 'f', kde->y, cs.pnk, 4);
  put("kde_z", 'f', kde->z, cs.pnk, 4);
  put("kde_t", 'i', kde->t, cs.pnk, 4);
  for (int m = 0; m < cs.pos; ++m) {
    put("mcs_x", 'f', mcs[m].x, MAXMCS, 4);
    put("mcs_y", 'f', mcs[m].y, MAXMCS, 4);
    put("mcs_z", 'f', mcs[m].z, MAXMCS, 4);
    put("mcs_tcc", 'f', &mcs[m].tcc, 1, 4);
  }
  fclose(g_out);
  printf("n_lig %d n_prt %d lna %d pnp %d pnk %d pos %d\n", cs.n_lig, cs.n_prt, cs.lna, cs.pnp,
         cs.pnk, cs.pos);
  return 0;
}
