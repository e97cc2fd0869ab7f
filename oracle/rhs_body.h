/*
 * Body of the oracle RHS, included twice by oracle.c: once with NUM = double and
 * once with NUM = double complex (complex-step derivatives in a and tau).
 * Restates model_synchronous (src/discoeb/perturbations.py:88-525) term by term.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */

static NUM FN(spl_eval)(const OracleSpline* s, NUM xn)
{
    int i = spline_index(s, RE(xn));
    double h = s->x[i + 1] - s->x[i];
    NUM t = (xn - s->x[i]) / h;
    NUM A = 1.0 - t, B = t;
    return A * s->y[i] + B * s->y[i + 1] + ((A * A * A - A) * s->S[i] + (B * B * B - B) * s->S[i + 1]) * (h * h) / 6.0;
}

static NUM FN(spl_deriv)(const OracleSpline* s, NUM xn)
{
    int i = spline_index(s, RE(xn));
    double h = s->x[i + 1] - s->x[i];
    NUM d = xn - s->x[i];
    double b = (s->y[i + 1] - s->y[i]) / h - h * (s->S[i + 1] + 2.0 * s->S[i]) / 6.0;
    double c = s->S[i] / 2.0;
    double dd = (s->S[i + 1] - s->S[i]) / (6.0 * h);
    return b + 2.0 * c * d + 3.0 * dd * d * d;
}

static NUM FN(maxr)(NUM x, double lo) { return RE(x) > lo ? x : (NUM)lo; }

static NUM FN(aprimeoa)(const OracleProblem* P, NUM a)
{
    NUM rhonu = EXP(FN(spl_eval)(&P->logrhonu_loga, LOG(a)));
    NUM rho_Q = POW(a, -3.0 * (1.0 + P->w0 + P->wa)) * EXP(3.0 * (a - 1.0) * P->wa);
    NUM grho = P->grhom * P->Omegam / a + (P->grhog + P->grhor * (P->Neff + P->Nmnu * rhonu)) / (a * a)
             + P->grhom * P->OmegaDE * rho_Q * a * a + P->grhom * P->Omegak;
    return SQRT(grho / 3.0);
}

static void FN(rhs)(const OracleProblem* P, NUM tau, const NUM* y, double kmode, NUM* f, int regime)
{
    const int lmaxg = P->lmaxg, lmaxgp = P->lmaxgp, lmaxr = P->lmaxr, lmaxnu = P->lmaxnu, nq = P->nqmax;
    const int n = P->n;
    const double Omegac = P->Omegam - P->Omegab;
    const int iq0 = 10 + lmaxg + lmaxgp + lmaxr, iq1 = iq0 + nq, iq2 = iq1 + nq, iq3 = iq2 + nq;
    const double k2 = kmode * kmode;
    const double s2_squared = 1.0, s_l2 = 1.0, s_l3 = 1.0;
    for (int i = 0; i < n; ++i) f[i] = 0.0;

    NUM a = y[0], loga = LOG(a), eta = y[2];
    NUM deltac = y[3], thetac = y[4], deltab = y[5], thetab = y[6];
    NUM deltag = y[7], thetag = y[8], shearg = y[9] / 2.0;
    NUM deltar = y[9 + lmaxg + lmaxgp], thetar = y[10 + lmaxg + lmaxgp], shearr = y[11 + lmaxg + lmaxgp] / 2.0;
    NUM deltaq = y[n - 2], thetaq = y[n - 1];

    NUM cs2 = FN(spl_eval)(&P->cs2a_loga, loga) / a;
    NUM xe = FN(spl_eval)(&P->xe_loga, loga);
    NUM photbar = P->grhog / (P->grhom * P->Omegab * a);
    NUM pb43 = 4.0 / 3.0 * photbar;
    NUM pnu = EXP(FN(spl_eval)(&P->logpnu_loga, loga));

    double cs2_Q = P->cs2_DE;
    NUM w_Q = P->w0 + P->wa * (1.0 - a);
    NUM rho_Q = POW(a, -3.0 * (1.0 + P->w0 + P->wa)) * EXP(3.0 * (a - 1.0) * P->wa);
    NUM rho_plus_p_theta_Q = (1.0 + w_Q) * rho_Q * P->grhom * P->OmegaDE * thetaq * a * a;

    NUM aprimeoa = FN(aprimeoa)(P, a);
    NUM xeprime = FN(spl_deriv)(&P->xe_loga, loga) * aprimeoa;
    NUM gpres = ((P->grhog + P->grhor * P->Neff) / 3.0 + P->grhor * P->Nmnu * pnu) / (a * a)
              + w_Q * P->grhom * P->OmegaDE * rho_Q * a * a;
    NUM aprimeprimeoa = 0.5 * (aprimeoa * aprimeoa - gpres);
    NUM w_Q_prime = -P->wa * aprimeoa * a;
    NUM ca2_Q = w_Q - w_Q_prime / 3.0 / ((1.0 + w_Q) + 1e-6) / aprimeoa;

    double akthom = 2.3038921003709498e-9 * (1.0 - P->YHe) * P->Omegab * P->H0 * P->H0;
    NUM opac = xe * akthom / (a * a);
    NUM tauc = 1.0 / FN(maxr)(opac, 1e-30);
    NUM taucprime = tauc * (2.0 * aprimeoa - xeprime / FN(maxr)(xe, 1e-30));
    NUM tauh = 1.0 / FN(maxr)(aprimeoa, 1e-30);
    double tauk = 1.0 / (kmode > 1e-30 ? kmode : 1e-30);

    int do_rsa, do_ufa, do_tca;
    if (regime < 0) {
        double tr = RE(tau), tcr = RE(tauc), thr = RE(tauh);
        do_rsa = P->use_rsa && (tcr / (tr > 1e-30 ? tr : 1e-30) > P->rsa_tau_c_over_tau) &&
                 (tr * kmode > P->rsa_tau_over_tau_k);
        do_ufa = !do_rsa && P->use_ufa && (tr * kmode > P->ufa_tau_over_tau_k);
        int uncoupled = (tcr / tauk > P->tca_tau_c_over_tau_k) ||
                        ((tcr / (thr > 1e-30 ? thr : 1e-30) > P->tca_tau_c_over_tau_h) &&
                         (tcr / tauk > 0.1 * P->tca_tau_c_over_tau_k));
        do_tca = !do_rsa && P->use_tca && !uncoupled;
    } else {
        do_rsa = (regime & 1) != 0;
        do_ufa = !do_rsa && (regime & 2) != 0;
        do_tca = !do_rsa && (regime & 4) != 0;
    }

    f[0] = aprimeoa * a;

    /* nu_perturb */
    NUM drhonu = 0.0, dpnu = 0.0, fnu = 0.0, shearnu = 0.0;
    NUM vq[ORACLE_MAX_NQ];
    for (int i = 0; i < nq; ++i) {
        NUM aq = a * P->amnu / P->q[i];
        NUM v = 1.0 / SQRT(1.0 + aq * aq);
        vq[i] = v;
        drhonu += P->w[i] * y[iq0 + i] / v;
        dpnu += P->w[i] * y[iq0 + i] * v;
        fnu += P->w[i] * y[iq1 + i];
        shearnu += P->w[i] * y[iq2 + i] * v;
    }
    dpnu /= 3.0;
    shearnu = shearnu * 2.0 / 3.0;

    NUM a2 = a * a;
    NUM dgrho = P->grhom * (Omegac * deltac + P->Omegab * deltab) / a
              + (P->grhog * deltag + P->grhor * (P->Neff * deltar + P->Nmnu * drhonu)) / a2
              + P->grhom * P->OmegaDE * deltaq * rho_Q * a2;
    NUM dgrho_wo_rel = P->grhom * (Omegac * deltac + P->Omegab * deltab) / a + P->grhor * P->Nmnu * drhonu / a2
                     + P->grhom * P->OmegaDE * deltaq * rho_Q * a2;
    NUM hprime_rsa = (2.0 * k2 * eta + dgrho_wo_rel) / FN(maxr)(aprimeoa, 1e-30);

    /* compute_fields_rsa (approximations.py:28-47) */
    double safe_k2 = k2 > 1e-30 ? k2 : 1e-30;
    NUM safe_tauc = FN(maxr)(tauc, 1e-30);
    NUM deltag_rsa = 4.0 / safe_k2 * (aprimeoa * hprime_rsa - safe_k2 * eta) +
                     4.0 / (safe_k2 * safe_tauc) * (thetab + 0.5 * hprime_rsa);
    NUM thetag_rsa = -0.5 * hprime_rsa + 3.0 / (safe_k2 * safe_tauc) *
                     (-taucprime / safe_tauc * (thetab + 0.5 * hprime_rsa) +
                      (-aprimeoa * thetab + cs2 * safe_k2 * deltab + safe_k2 * eta));
    NUM deltar_rsa = 4.0 / safe_k2 * (aprimeoa * hprime_rsa - safe_k2 * eta);
    NUM thetar_rsa = -0.5 * hprime_rsa;

    NUM deltag_eff = do_rsa ? deltag_rsa : deltag;
    NUM thetag_eff = do_rsa ? thetag_rsa : thetag;
    NUM shearg_eff = do_rsa ? (NUM)0.0 : shearg;
    NUM deltar_eff = do_rsa ? deltar_rsa : deltar;
    NUM thetar_eff = do_rsa ? thetar_rsa : thetar;
    NUM shearr_eff = do_rsa ? (NUM)0.0 : shearr;

    NUM dgpres = (P->grhog * deltag_eff + P->grhor * P->Neff * deltar_eff) / a2 / 3.0 +
                 P->grhor * P->Nmnu * dpnu / a2 +
                 (cs2_Q * P->grhom * P->OmegaDE * deltaq * rho_Q * a2 +
                  (cs2_Q - ca2_Q) * (3.0 * aprimeoa * rho_plus_p_theta_Q / k2));
    NUM dgtheta = P->grhom * (Omegac * thetac + P->Omegab * thetab) / a +
                  4.0 / 3.0 * (P->grhog * thetag_eff + P->Neff * P->grhor * thetar_eff) / a2 +
                  P->Nmnu * P->grhor * kmode * fnu / a2 + rho_plus_p_theta_Q;
    (void)shearnu;

    f[1] = -(dgrho + 3.0 * dgpres) * a;
    NUM hprime_full = (2.0 * k2 * eta + dgrho) / aprimeoa;
    NUM hprime = do_rsa ? hprime_rsa : hprime_full;
    NUM etaprime = 0.5 * dgtheta / k2;
    NUM alpha = (hprime + 6.0 * etaprime) / 2.0 / k2;
    f[2] = etaprime;
    f[3] = -thetac - 0.5 * hprime;
    f[4] = -aprimeoa * thetac;
    const int idxb = 5;
    f[idxb] = -thetab - 0.5 * hprime;
    f[idxb + 1] = -aprimeoa * thetab + k2 * cs2 * deltab + pb43 * opac * (thetag_eff - thetab);

    const int idxg = 7, idxgp = 7 + (lmaxg + 1);
    if (do_rsa) {
        /* photon entries stay zero */
    } else if (do_tca) {
        NUM deltabprime_tca = -thetab - 0.5 * hprime;
        NUM thetabprime_tca = (-aprimeoa * thetab + k2 * cs2 * deltab +
                               k2 * pb43 * (0.25 * deltag - s2_squared * shearg)) / (1.0 + pb43);
        NUM deltagprime_tca = 4.0 / 3.0 * (-thetag - 0.5 * hprime);
        NUM slip = 2.0 * pb43 / (1.0 + pb43) * aprimeoa * (thetab - thetag) +
                   tauc * (-aprimeprimeoa * thetab - 0.5 * aprimeoa * k2 * deltag +
                           k2 * (cs2 * deltabprime_tca - 0.25 * deltagprime_tca)) / (1.0 + pb43);
        thetabprime_tca = thetabprime_tca + pb43 / (1.0 + pb43) * slip;
        NUM thetagprime_tca = (-thetabprime_tca - aprimeoa * thetab + k2 * cs2 * deltab) / FN(maxr)(pb43, 1e-30) +
                              k2 * (0.25 * deltag - s2_squared * shearg);
        f[idxb] = deltabprime_tca;
        f[idxb + 1] = thetabprime_tca;
        f[idxg] = deltagprime_tca;
        f[idxg + 1] = thetagprime_tca;
    } else {
        NUM polter = y[idxg + 2] + y[idxgp + 0] + y[idxgp + 2];
        f[idxg] = 4.0 / 3.0 * (-thetag_eff - 0.5 * hprime);
        f[idxg + 1] = k2 * (0.25 * deltag_eff - s2_squared * shearg_eff) - opac * (thetag_eff - thetab);
        f[idxg + 2] = 8.0 / 15.0 * (thetag_eff + k2 * alpha) - 3.0 / 5.0 * kmode * s_l3 / s_l2 * y[idxg + 3] -
                      opac * (y[idxg + 2] - 0.1 * s_l2 * polter);
        for (int l = 3; l < lmaxg; ++l)
            f[idxg + l] = kmode / (2 * l + 1) * (l * y[idxg + l - 1] - (l + 1) * y[idxg + l + 1]) - opac * y[idxg + l];
        f[idxg + lmaxg] = kmode * y[idxg + lmaxg - 1] - (lmaxg + 1) / tau * y[idxg + lmaxg] - opac * y[idxg + lmaxg];
        for (int l = 0; l < lmaxgp; ++l) {
            NUM lower = (l == 0) ? (NUM)0.0 : l * y[idxgp + l - 1];
            f[idxgp + l] = kmode / (2 * l + 1) * (lower - (l + 1) * y[idxgp + l + 1]) - opac * y[idxgp + l];
        }
        f[idxgp + 0] += opac * polter / 2.0;
        f[idxgp + 2] += opac * polter / 10.0;
        f[idxgp + lmaxgp] = kmode * y[idxgp + lmaxgp - 1] - (lmaxgp + 1) / tau * y[idxgp + lmaxgp] - opac * y[idxgp + lmaxgp];
    }

    const int idxr = 9 + lmaxg + lmaxgp;
    if (do_rsa) {
        /* massless neutrino entries stay zero */
    } else {
        f[idxr] = 4.0 / 3.0 * (-thetar_eff - 0.5 * hprime);
        f[idxr + 1] = k2 * (0.25 * deltar_eff - shearr_eff);
        if (do_ufa) {
            f[idxr + 2] = -3.0 / FN(maxr)(tau, 1e-30) * shearr_eff + 4.0 / 15.0 * (thetar_eff + 0.5 * hprime);
        } else {
            f[idxr + 2] = 8.0 / 15.0 * (thetar_eff + k2 * alpha) - 0.6 * kmode * y[idxr + 3];
            for (int l = 3; l < lmaxr; ++l)
                f[idxr + l] = kmode / (2 * l + 1) * (l * y[idxr + l - 1] - (l + 1) * y[idxr + l + 1]);
            f[idxr + lmaxr] = kmode * y[idxr + lmaxr - 1] - (lmaxr + 1) / tau * y[idxr + lmaxr];
        }
    }

    for (int i = 0; i < nq; ++i) {
        double qi = P->q[i];
        double dlfdlq = -qi / (1.0 + exp(-qi));
        NUM v = vq[i];
        f[iq0 + i] = -kmode * v * y[iq1 + i] + hprime * dlfdlq / 6.0;
        f[iq1 + i] = kmode * v * (y[iq0 + i] - 2.0 * y[iq2 + i]) / 3.0;
        f[iq2 + i] = kmode * v * (2.0 * y[iq1 + i] - 3.0 * y[iq3 + i]) / 5.0 - (hprime / 15.0 + 2.0 / 5.0 * etaprime) * dlfdlq;
        for (int l = 3; l < lmaxnu; ++l)
            f[iq0 + l * nq + i] = kmode * v / (2 * l + 1) *
                                  (l * y[iq0 + (l - 1) * nq + i] - (l + 1) * y[iq0 + (l + 1) * nq + i]);
        f[iq0 + lmaxnu * nq + i] = kmode * v * y[iq0 + (lmaxnu - 1) * nq + i] - (lmaxnu + 1) / tau * y[iq0 + lmaxnu * nq + i];
    }

    if (P->de_guard_eps > 0.0 && fabs(RE(1.0 + w_Q)) < P->de_guard_eps) {
        f[n - 2] = 0.0;
        f[n - 1] = 0.0;
    } else {
        f[n - 2] = -(1.0 + w_Q) * (thetaq + 0.5 * hprime) - 3.0 * (cs2_Q - w_Q) * aprimeoa * deltaq -
                   9.0 * (1.0 + w_Q) * (cs2_Q - ca2_Q) * aprimeoa * aprimeoa / k2 * thetaq;
        f[n - 1] = -(1.0 - 3.0 * cs2_Q) * aprimeoa * thetaq + cs2_Q / (1.0 + w_Q) * k2 * deltaq;
    }
}
