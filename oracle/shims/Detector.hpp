/*
 * Test-infrastructure shim (oracle only): stands in for the lisatools C++ header
 * `Detector.hpp` that the reference's Response.cu includes (Response.cu:6) and that
 * the reference copies in from the external lisaanalysistools package at build time.
 * That package is not available here, so this header supplies the interface the
 * response code uses:
 *   Orbits::get_pos(t, sc)               (Response.cu:86-98)
 *   Orbits::get_normal_unit_vec(t, link) (Response.cu:103-127)
 *   Orbits::armlength                    (Response.cu:169-173, 205)
 *   AddOrbits::add_orbit_information(dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e,
 *                                    armlength), AddOrbits::dealloc()
 *                                         (signature: lisaresponse.pyx:12-13)
 *
 * Table layout and lookup rule (shared bit-for-bit with the bbhx_b200 product so both
 * read identical orbits):
 *   x_arr[N][3][3]   spacecraft positions (m), spacecraft 1..3, xyz
 *   n_arr[N][6][3]   link unit vectors, link order given by links[6] (e.g. 12,23,31,13,32,21)
 *   L_arr[N][6]      link lengths (m)
 *   sample k sits at t = k*dt.  A query at time t uses window w = floor(t/dt); when
 *   0 <= w < N-1 the value is down + (up - down)/dt * (t - w*dt) per component,
 *   otherwise the zero vector is returned.
 */
#ifndef ORACLE_SHIM_DETECTOR_HPP
#define ORACLE_SHIM_DETECTOR_HPP

#include <cmath>
#include <stdexcept>

class Vec
{
public:
    double x, y, z;
    Vec(double x_ = 0.0, double y_ = 0.0, double z_ = 0.0) : x(x_), y(y_), z(z_) {}
};

class Orbits
{
public:
    double dt = 0.0;
    int N = 0;
    double *n_arr = nullptr;
    double *L_arr = nullptr;
    double *x_arr = nullptr;
    int links[6] = {0, 0, 0, 0, 0, 0};
    int sc_r[6] = {0, 0, 0, 0, 0, 0};
    int sc_e[6] = {0, 0, 0, 0, 0, 0};
    double armlength = 0.0;

    int window(double t) const
    {
        double w = std::floor(t / dt);
        if (!(w >= 0.0) || w >= (double)(N - 1))
            return -1;
        return (int)w;
    }

    int link_index(int link) const
    {
        for (int i = 0; i < 6; i++)
            if (links[i] == link)
                return i;
        return -1;
    }

    Vec lerp3(const double *tab, int stride, int offset, double t) const
    {
        int w = window(t);
        if (w < 0)
            return Vec(0.0, 0.0, 0.0);
        const double *lo = tab + (size_t)w * stride + offset;
        const double *hi = tab + (size_t)(w + 1) * stride + offset;
        double tt = t - w * dt;
        return Vec(lo[0] + (hi[0] - lo[0]) / dt * tt,
                   lo[1] + (hi[1] - lo[1]) / dt * tt,
                   lo[2] + (hi[2] - lo[2]) / dt * tt);
    }

    Vec get_pos(double t, int sc) const { return lerp3(x_arr, 9, (sc - 1) * 3, t); }

    Vec get_normal_unit_vec(double t, int link) const
    {
        int li = link_index(link);
        if (li < 0)
            return Vec(0.0, 0.0, 0.0);
        return lerp3(n_arr, 18, li * 3, t);
    }
};

class AddOrbits
{
public:
    Orbits *orbits = nullptr;

    void add_orbit_information(double dt_, int N_, double *n_arr_, double *L_arr_, double *x_arr_,
                               int *links_, int *sc_r_, int *sc_e_, double armlength_)
    {
        if (orbits == nullptr)
            orbits = new Orbits();
        orbits->dt = dt_;
        orbits->N = N_;
        orbits->n_arr = n_arr_;
        orbits->L_arr = L_arr_;
        orbits->x_arr = x_arr_;
        for (int i = 0; i < 6; i++)
        {
            orbits->links[i] = links_[i];
            orbits->sc_r[i] = sc_r_[i];
            orbits->sc_e[i] = sc_e_[i];
        }
        orbits->armlength = armlength_;
    }

    void dealloc()
    {
        delete orbits;
        orbits = nullptr;
    }
};

#endif
