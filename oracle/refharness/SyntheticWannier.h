/* SyntheticWannier -- harness-only material for the reference build.
 *
 * TEST INFRASTRUCTURE: compiled only into oracle/_ref/exec_hhg_harness (see
 * oracle/make_harness.py and oracle/Makefile), where the reference's own
 * SBEs class propagates it.  It is never part of the product.
 *
 * An N-band tight-binding model in the model form of the reference's
 * Materials/Wannier90.h:297-387, with explicit tables instead of a Wannier90
 * file, read from the cfg group of the same name:
 *
 *   SyntheticWannier = { Nband; Nval; lattice = [a1x, a1y, a2x, a2y];
 *                        R = [n1, n2, ...]; h_re, h_im  [nR][N][N];
 *                        d_re, d_im [nR][2][N][N] (optional) };
 *
 *   H(k)   = sum_R h_R e^{i k.R}             R = n1 a1 + n2 a2 (bohr)
 *   D_a(k) = sum_R d_{a,R} e^{i k.R}         a = x, y; D_z = 0
 *   J_a(k) = -dH/dk_a + i [D_a(k), H(k)]     BaseMaterial.h:62-68; J_z = 0
 *
 * isDipoleZero is false when dipole tables are given, so the reference's
 * length gauge adds E(t).D(k+A) to H0(k+A) (SBEs.h:771-782) and its currents
 * use the full J of BaseMaterial.h.  The Brillouin zone is spanned by the
 * reciprocal basis b_i . a_j = 2 pi delta_ij with origin 0.  The sums run
 * over R in table order, elements innermost, the order the C oracle uses.
 */
#pragma once

#include <array>
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <tuple>
#include <vector>

#include <libconfig.h++>

#include "BaseMaterial.h"

class SyntheticWannier : public BaseMaterial
{
public:
    int nR;
    double lattice[4];
    std::vector<double> Rc;       // [nR][2] Cartesian lattice vectors
    std::vector<complex> hR;      // [nR][N*N]
    std::vector<complex> dR;      // [nR][2][N*N], empty without dipoles

    explicit SyntheticWannier(const libconfig::Setting *_cfg)
    {
        const libconfig::Setting &cfg = *_cfg;
        if (!cfg.lookupValue("Nband", Nband) || !cfg.lookupValue("Nval", Nval))
        {
            std::cerr << "SyntheticWannier: Nband and Nval are required\n";
            std::exit(EXIT_FAILURE);
        }
        const libconfig::Setting &lat = cfg["lattice"];
        for (int i = 0; i < 4; ++i) lattice[i] = lat[i];
        const libconfig::Setting &R = cfg["R"];
        nR = R.getLength() / 2;
        const int NN = Nband * Nband;
        Rc.resize(2 * (size_t)nR);
        for (int r = 0; r < nR; ++r)
        {
            const int n1 = R[2 * r], n2 = R[2 * r + 1];
            Rc[2 * r]     = n1 * lattice[0] + n2 * lattice[2];
            Rc[2 * r + 1] = n1 * lattice[1] + n2 * lattice[3];
        }
        const libconfig::Setting &hre = cfg["h_re"], &him = cfg["h_im"];
        if (hre.getLength() != nR * NN || him.getLength() != nR * NN)
        {
            std::cerr << "SyntheticWannier: h_re / h_im must hold nR*N*N values\n";
            std::exit(EXIT_FAILURE);
        }
        hR.resize((size_t)nR * NN);
        for (int i = 0; i < nR * NN; ++i) hR[i] = complex((double)hre[i], (double)him[i]);
        isDipoleZero = !cfg.exists("d_re");
        if (!isDipoleZero)
        {
            const libconfig::Setting &dre = cfg["d_re"], &dim = cfg["d_im"];
            if (dre.getLength() != 2 * nR * NN || dim.getLength() != 2 * nR * NN)
            {
                std::cerr << "SyntheticWannier: d_re / d_im must hold nR*2*N*N values\n";
                std::exit(EXIT_FAILURE);
            }
            dR.resize(2 * (size_t)nR * NN);
            for (int i = 0; i < 2 * nR * NN; ++i) dR[i] = complex((double)dre[i], (double)dim[i]);
        }
    }

    // H and both derivatives dH/dk_a in one pass over R
    void Synthesize(complex *H, complex *dHx, complex *dHy, complex *Dx, complex *Dy,
                    const std::array<double, Ndim> &k) const
    {
        const int NN = Nband * Nband;
        for (int i = 0; i < NN; ++i)
        {
            H[i] = 0.;
            if (dHx) { dHx[i] = 0.; dHy[i] = 0.; }
            if (Dx) { Dx[i] = 0.; Dy[i] = 0.; }
        }
        for (int r = 0; r < nR; ++r)
        {
            const double ph = k[0] * Rc[2 * r] + k[1] * Rc[2 * r + 1];
            const complex e(std::cos(ph), std::sin(ph));
            for (int i = 0; i < NN; ++i)
            {
                const complex hv = hR[(size_t)r * NN + i] * e;
                H[i] += hv;
                if (dHx)
                {
                    dHx[i] += I * Rc[2 * r] * hv;
                    dHy[i] += I * Rc[2 * r + 1] * hv;
                }
            }
            if (Dx && !isDipoleZero)
            {
                for (int i = 0; i < NN; ++i)
                {
                    Dx[i] += dR[((size_t)r * 2 + 0) * NN + i] * e;
                    Dy[i] += dR[((size_t)r * 2 + 1) * NN + i] * e;
                }
            }
        }
    }

    void GenHamiltonian(complex *_hstore, std::array<double, Ndim> _kpoint) override
    {
        Synthesize(_hstore, nullptr, nullptr, nullptr, nullptr, _kpoint);
    }

    void GenDipole(complex **_dstore, std::array<double, Ndim> _kpoint) override
    {
        const int NN = Nband * Nband;
        std::vector<complex> H(NN);
        for (int i = 0; i < NN; ++i) _dstore[2][i] = 0.;
        if (isDipoleZero)
        {
            for (int i = 0; i < NN; ++i) { _dstore[0][i] = 0.; _dstore[1][i] = 0.; }
            return;
        }
        Synthesize(H.data(), nullptr, nullptr, _dstore[0], _dstore[1], _kpoint);
    }

    void GenJMatrix(complex **_jstore, std::array<double, Ndim> _kpoint) override
    {
        const int N = Nband, NN = N * N;
        std::vector<complex> H(NN), dH(2 * NN), D(2 * NN);
        Synthesize(H.data(), dH.data(), dH.data() + NN, D.data(), D.data() + NN, _kpoint);
        for (int a = 0; a < 2; ++a)
        {
            for (int i = 0; i < N; ++i)
            {
                for (int j = 0; j < N; ++j)
                {
                    complex v = -dH[a * NN + i * N + j];
                    if (!isDipoleZero)
                    {
                        complex c = 0.;
                        for (int l = 0; l < N; ++l)
                            c += D[a * NN + i * N + l] * H[l * N + j] - H[i * N + l] * D[a * NN + l * N + j];
                        v += I * c;
                    }
                    _jstore[a][i * N + j] = v;
                }
            }
        }
        for (int i = 0; i < NN; ++i) _jstore[2][i] = 0.;
    }

    std::tuple<std::array<double, Ndim * Ndim>, std::array<double, Ndim>> GenBrillouinzone() override
    {
        const double det = lattice[0] * lattice[3] - lattice[1] * lattice[2];
        std::array<double, Ndim * Ndim> axes = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
        axes[0] = 2 * M_PI * lattice[3] / det;
        axes[1] = -2 * M_PI * lattice[2] / det;
        axes[3] = -2 * M_PI * lattice[1] / det;
        axes[4] = 2 * M_PI * lattice[0] / det;
        std::array<double, Ndim> origin = {0., 0., 0.};
        return std::make_tuple(axes, origin);
    }

    void PrintMaterialInformation() override
    {
        std::cout << "SyntheticWannier (harness): Nband = " << Nband << ", Nval = " << Nval
                  << ", nR = " << nR << ", dipoles " << (isDipoleZero ? "off" : "on") << "\n";
    }
};
