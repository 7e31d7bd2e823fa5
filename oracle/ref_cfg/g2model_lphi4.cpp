/*
 * lambda phi^4 + g^2 phi^2 chi^2 model for the reference build.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference ships one model file
 * (g2model.cpp: m^2 phi^2/2 + g^2 phi^2 chi^2/2) and tells users to edit it
 * for other models (g2model.cpp:5-19).  The preheating configurations use
 * V = lambda phi^4/4 + g^2 phi^2 chi^2/2, so this file supplies the same five
 * entry points (modelinfo, potential, dVdf, effMass, initfields; reference
 * g2model.cpp:32-144) for that potential, written in the reference's
 * rescaling (x_pr = B x, t_pr = B t, f_pr = f, V_pr = V/B^2, B =
 * sqrt(lambda) phi0):
 *
 *   V_pr   = lam_pr phi^4/4 + gsq_pr phi^2 chi^2/2
 *   dV/dphi = lam_pr phi^3 + gsq_pr chi^2 phi
 *   dV/dchi = gsq_pr phi^2 chi
 *   m_eff^2(phi) = <3 lam_pr phi^2 + gsq_pr chi^2>,  m_eff^2(chi) = <gsq_pr phi^2>
 *
 * The order of floating-point operations in potential/dVdf is the one the
 * CUDA kernels and oracle/gabe_oracle.c use, so FP64 results can agree to the
 * last bit.  initfields follows the reference's two-call protocol
 * (g2model.cpp:113-144): call 0 sets the homogeneous values, call 1 adds the
 * random fluctuations field by field, each call ends with calcEnergy(0).
 */
#include "g2header.h"

void modelinfo(FILE *info)
{
    fprintf(info, "lambda phi^4 preheating\n");
    fprintf(info, "V = lambda/4 phi^4 + g^2/2 phi^2 chi^2\n\n");
    fprintf(info, "lambda= %e\n", lambda_phys);
    fprintf(info, "g^2/lambda= %e\n", g2_over_lambda);
    fprintf(info, "phi0= %e m_pl, dphi0= %e\n", f0[0], df0[0]);
    fprintf(info, "Using random initial conditions");
}

gNum potential(int s, int i, int j, int k)
{
    const gNum p = field[s][0][i][j][k];
    const gNum c = field[s][1][i][j][k];
    return 0.25 * lam_pr * p * p * p * p + 0.5 * gsq_pr * p * p * c * c;
}

gNum dVdf(int s, int fld, int i, int j, int k)
{
    const gNum p = field[s][0][i][j][k];
    const gNum c = field[s][1][i][j][k];
    if (fld == 0) return lam_pr * p * p * p + gsq_pr * c * c * p;
    if (fld == 1) return gsq_pr * p * p * c;
    return 0.;
}

inline gNum effMass(int s, int fld)
{
    gNum m2 = 0.;
    int i, j, k;
    if (fld == 0) {
        LOOP { m2 += 3. * lam_pr * field[s][0][i][j][k] * field[s][0][i][j][k]
                     + gsq_pr * field[s][1][i][j][k] * field[s][1][i][j][k]; }
        return m2 / gridsize;
    }
    if (fld == 1) {
        LOOP { m2 += gsq_pr * field[s][0][i][j][k] * field[s][0][i][j][k]; }
        return m2 / gridsize;
    }
    return 1.;
}

void initfields()
{
    static int call = 0;
    const int s = 0;
    DECLARE_INDEX
    if (call == 0) {
        fldLOOP {
            field[s][fld][i][j][k] = f0[fld];
            dfield[s][fld][i][j][k] = df0[fld];
        }
    }
    if (call == 1) {
        for (fld = 0; fld < nflds; fld++)
            randInit(field[s][fld], dfield[s][fld], effMass(s, fld));
        initDestroy();
    }
    calcEnergy(0);
    call++;
}
