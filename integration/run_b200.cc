// run_b200.cc -- Run() of gpudocksm-rem-1.2/src/run.h on the B200 library.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include "dock.h"
#include "run.h"
#include "toggle.h"
#include "gpudock.h"

static_assert(sizeof(EnePara) == sizeof(gd_enepara), "EnePara and gd_enepara must match");

void Run(const Ligand *lig, const Protein *prt, const Psp *psp, const Kde *kde, const Mcs *mcs,
         const EnePara *enepara, const Temp *temp, const Replica *replica, const McPara *mcpara,
         McLog *mclog, const ComplexSize cs) {
  (void)replica;  // the flat layout n_tmp*n_lig*p + n_lig*t + l is implied
  const int lna = cs.lna, pnp = cs.pnp, n_lig = cs.n_lig, n_prt = cs.n_prt;
  std::vector<float> lx(n_lig * lna), ly(n_lig * lna), lz(n_lig * lna);
  for (int l = 0; l < n_lig; ++l)  // replicas 0..n_lig-1 hold the conformations
    for (int a = 0; a < lna; ++a) {
      lx[l * lna + a] = lig[l].coord_orig.x[a];
      ly[l * lna + a] = lig[l].coord_orig.y[a];
      lz[l * lna + a] = lig[l].coord_orig.z[a];
    }
  std::vector<float> px(n_prt * pnp), py(n_prt * pnp), pz(n_prt * pnp);
  for (int p = 0; p < n_prt; ++p)
    for (int i = 0; i < pnp; ++i) {
      px[p * pnp + i] = prt[p].x[i];
      py[p * pnp + i] = prt[p].y[i];
      pz[p * pnp + i] = prt[p].z[i];
    }
  std::vector<float> mx(cs.pos * MAXMCS), my(cs.pos * MAXMCS), mz(cs.pos * MAXMCS), tcc(cs.pos);
  for (int m = 0; m < cs.pos; ++m) {
    std::memcpy(&mx[m * MAXMCS], mcs[m].x, sizeof(float) * MAXMCS);
    std::memcpy(&my[m * MAXMCS], mcs[m].y, sizeof(float) * MAXMCS);
    std::memcpy(&mz[m * MAXMCS], mcs[m].z, sizeof(float) * MAXMCS);
    tcc[m] = mcs[m].tcc;
  }
  gd_complex cx;
  std::memset(&cx, 0, sizeof(cx));
  cx.lig.lna = lna;
  cx.lig.n_conf = n_lig;
  cx.lig.x = lx.data();
  cx.lig.y = ly.data();
  cx.lig.z = lz.data();
  cx.lig.t = lig[0].t;
  cx.lig.c = lig[0].c;
  cx.lig.n = lig[0].n;
  std::memcpy(cx.lig.center, lig[0].coord_orig.center, sizeof(cx.lig.center));
  cx.prt.pnp = pnp;
  cx.prt.n_conf = n_prt;
  cx.prt.x = px.data();
  cx.prt.y = py.data();
  cx.prt.z = pz.data();
  cx.prt.t = prt[0].t;
  cx.prt.c = prt[0].c;
  cx.prt.ele = prt[0].ele;
  cx.prt.seq3r = prt[0].seq3r;
  cx.prt.c0_and_d12_or_c2 = prt[0].c0_and_d12_or_c2;
  cx.prt.hpp = prt[0].hpp;
  std::memcpy(cx.prt.pocket_center, prt[0].pocket_center, sizeof(cx.prt.pocket_center));
  cx.psp.n_col = MAXPRO;
  cx.psp.psp = &psp->psp[0][0];
  cx.kde.pnk = cs.pnk;
  cx.kde.x = kde->x;
  cx.kde.y = kde->y;
  cx.kde.z = kde->z;
  cx.kde.t = kde->t;
  cx.mcs.pos = cs.pos;
  cx.mcs.n_field = MAXMCS;
  cx.mcs.x = mx.data();
  cx.mcs.y = my.data();
  cx.mcs.z = mz.data();
  cx.mcs.tcc = tcc.data();
  cx.ff = reinterpret_cast<const gd_enepara *>(enepara);

  std::vector<float> mb(cs.n_tmp);
  for (int t = 0; t < cs.n_tmp; ++t) mb[t] = temp[t].minus_beta;
  gd_mc_params mc;
  std::memset(&mc, 0, sizeof(mc));
  mc.steps_total = mcpara->steps_total;
  mc.steps_per_exchange = mcpara->steps_per_exchange;
  mc.steps_per_dump = mcpara->steps_per_dump;
  mc.n_tmp = cs.n_tmp;
  std::memcpy(mc.move_scale, mcpara->move_scale, sizeof(mc.move_scale));
  mc.minus_beta = mb.data();
  mc.seed = (uint64_t)time(NULL);  // the reference seeds from the clock too
  mc.flags = GD_MC_EXCHANGE | (IS_AWAY ? GD_MC_MOVE_AWAY : 0) | (IS_CALCU_MCC ? GD_MC_MCC : 0) |
             (IS_BAYE ? GD_MC_BAYES : 0);

  std::vector<int> acs(cs.n_rep), acx(cs.n_tmp);
  gd_mc_log log;
  std::memset(&log, 0, sizeof(log));
  log.acs_mc = acs.data();
  log.acs_temp_exchg = acx.data();
  if (gd_run(&cx, &mc, &log) != GD_OK) {
    fprintf(stderr, "gd_run: %s\n", gd_last_error());
    exit(1);  // the reference's own failure behaviour
  }
  mclog->t0 = log.t_compute;
  mclog->t1 = log.t_wall;
  for (int r = 0; r < cs.n_rep && r < MAXREP; ++r) mclog->acs_mc[r] += acs[r];
  for (int t = 0; t < cs.n_tmp && t < MAXREP; ++t) mclog->acs_temp_exchg[t] += acx[t];
  mclog->ac_mc += (int)log.ac_mc;
  mclog->ac_temp_exchg += (int)log.ac_temp_exchg;
}
