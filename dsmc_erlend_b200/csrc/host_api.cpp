// host_api.cpp - host-only entry points of the C ABI: reference defaults,
// Setup() constants, WallModelName(), status strings and the field writer.
// Compiled with -ffp-contract=off so the derived constants are the IEEE
// sequence of the reference expressions.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <limits>
#include <string>

#include "../../include/dsmc.h"

namespace {
constexpr double K_BOLTZMANN = 1.380662E-23; // include/Constants.h:9
constexpr double N_AVOGADRO = 6.022045E+23;  // include/Constants.h:10
constexpr double PI_D = 3.14159265358979323846;

bool cll_valid(double an, double at)
{
    return std::isfinite(an) && an >= 0.0 && an <= 1.0 && std::isfinite(at) && at >= 0.0 &&
           at <= 1.0;
}

// The Gamma function of x > 0 with the reference's arithmetic
// (src/Initialization.cpp:111-207), so that CrRef and the free-stream mean
// free time and path come out with the same bits.  The method is the
// published one that code follows:
//   * x < 0.001: 1/Gamma(x) = x (1 + g x) + O(x^3), g = Euler's constant;
//   * 0.001 <= x < 12: W. J. Cody's rational approximation of Gamma on
//     (1, 2) (SPECFUN, Gamma(1 + z) = 1 + z P(z) / Q(z), the degree-8
//     numerator and denominator of Cody's published table, evaluated by
//     Horner's rule), then Gamma(x) = Gamma(x + 1) / x below 1 and the
//     recurrence Gamma(x + 1) = x Gamma(x) above 2;
//   * x >= 12: Stirling's series for log Gamma (Abramowitz and Stegun 6.1.41)
//     with the first eight Bernoulli terms, infinity beyond 171.624.
// Every operation is in the same order as there (this file is compiled
// without contraction into fused multiply-adds).
double gamma_ref(double x)
{
    constexpr double euler_gamma = 0.577215664901532860606512090;
    if (x < 0.001)
        return 1.0 / (x * (1.0 + euler_gamma * x));
    if (x < 12.0) {
        static const double num_coef[8] = {
            -1.71618513886549492533811E+0, 2.47656508055759199108314E+1,
            -3.79804256470945635097577E+2, 6.29331155312818442661052E+2,
            8.66966202790413211295064E+2,  -3.14512729688483675254357E+4,
            -3.61444134186911729807069E+4, 6.64561438202405440627855E+4};
        static const double den_coef[8] = {
            -3.08402300119738975254353E+1, 3.15350626979604161529144E+2,
            -1.01515636749021914166146E+3, -3.10777167157231109440444E+3,
            2.25381184209801510330112E+4,  4.75584627752788110767815E+3,
            -1.34659959864969306392456E+5, -1.15132259675553483497211E+5};
        const bool below_one = x < 1.0;
        int shift = 0; // recurrence steps from (1, 2) back up to x
        double y = x;
        if (below_one) {
            y += 1.0;
        } else {
            shift = static_cast<int>(std::floor(y)) - 1;
            y -= shift;
        }
        const double z = y - 1;
        double num = 0.0, den = 1.0;
        for (int i = 0; i < 8; ++i) {
            num = (num + num_coef[i]) * z;
            den = den * z + den_coef[i];
        }
        double g = num / den + 1.0;
        if (below_one) {
            g /= (y - 1.0);
        } else {
            for (int i = 0; i < shift; ++i)
                g *= y++;
        }
        return g;
    }
    if (x > 171.624)
        return std::numeric_limits<double>::max() * 2.0;
    static const double bern[8] = {1.0 / 12.0,   -1.0 / 360.0,      1.0 / 1260.0,
                                   -1.0 / 1680.0, 1.0 / 1188.0,      -691.0 / 360360.0,
                                   1.0 / 156.0,  -3617.0 / 122400.0};
    const double z = 1.0 / (x * x);
    double sum = bern[7];
    for (int i = 6; i >= 0; --i) {
        sum *= z;
        sum += bern[i];
    }
    const double series = sum / x;
    constexpr double half_log_2pi = 0.91893853320467274178032973640562;
    return std::exp((x - 0.5) * std::log(x) - x + half_log_2pi + series);
}
} // namespace

extern "C" {

void dsmc_default_params(dsmc_params *p)
{
    *p = dsmc_params{};
    // src/Geometry.cpp:11-24
    p->x1 = -20.0;
    p->x2 = 20.0;
    p->y1 = -20.0;
    p->y2 = 20.0;
    p->dz = 0.1;
    p->nx = 100;
    p->ny = 100;
    p->dl = 0.1;
    p->box_x = 0.0;
    p->box_y = 0.0;
    p->box_width = 4.0;
    p->box_height = 4.0;
    // src/Initialization.cpp:11-31
    p->dt = 1.0e-05;
    p->n_step = 100000;
    p->first_sampling_step = 10000;
    p->sampling_period = 1;
    p->npc_free = 10;
    p->molar_mass = 0.040;
    p->ma_free = 4;
    p->n_free = 1e17;
    p->t_free = 200;
    p->attack_angle = 0;
    p->t_wall = 300.0;
    p->d_ref = 4.17e-10;
    p->viscosity_index = 0.81;
    p->t_ref = 273.0;
    // src/Boundary.cpp:11-13
    p->wall_model = DSMC_WALL_CLL;
    p->cll_normal = 0.8;
    p->cll_tangential = 0.8;
    p->seed = 0x5EED;
    p->precision = DSMC_FP64;
}

// Setup(), src/Initialization.cpp:210-265, with the reference's Gamma
// (gamma_ref above): every derived constant has the reference's bits.
int dsmc_setup(const dsmc_params *p, dsmc_derived *d)
{
    if (p == nullptr || d == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (p->wall_model < DSMC_WALL_DIFFUSE || p->wall_model > DSMC_WALL_CLL)
        return DSMC_ERR_ARGUMENT;
    if (p->wall_model == DSMC_WALL_CLL && !cll_valid(p->cll_normal, p->cll_tangential))
        return DSMC_ERR_BAD_CLL;
    if (p->nx < 1 || p->ny < 1 || !(p->x2 > p->x1) || !(p->y2 > p->y1) || !(p->dt > 0.0) ||
        p->sampling_period < 1 || !(p->npc_free > 0.0) || !(p->dz > 0.0) ||
        p->precision < DSMC_FP64 || p->precision > DSMC_FP32 || p->reserved1 != 0)
        return DSMC_ERR_ARGUMENT;
    const double k = K_BOLTZMANN;
    d->molecule_mass = p->molar_mass / N_AVOGADRO;
    const double m = d->molecule_mass;
    d->p_free = p->n_free * (k * p->t_free);
    d->u_free = p->ma_free * std::sqrt((5.0 / 3.0) * k * p->t_free / m);
    d->ux_free = d->u_free * std::cos(PI_D * p->attack_angle / 180.0);
    d->uy_free = -d->u_free * std::sin(PI_D * p->attack_angle / 180.0);
    d->dx = (p->x2 - p->x1) / p->nx;
    d->dy = (p->y2 - p->y1) / p->ny;
    d->dv = d->dx * d->dy * p->dz;
    d->weight = d->dv * p->n_free / p->npc_free;
    d->sigma_ref = PI_D * p->d_ref * p->d_ref;
    d->omega = 2.0 * p->viscosity_index - 1.0;
    d->cr_ref = std::sqrt(4.0 * k * p->t_ref / m) /
                std::pow(gamma_ref(2.5 - p->viscosity_index), 1.0 / d->omega);
    const double q = 1.0 - d->omega;
    const double mean_rel = std::pow(4.0 * k * p->t_free / m, q / 2.0) *
                            gamma_ref((q + 3.0) / 2.0) / gamma_ref(1.5);
    const double rate = d->sigma_ref * std::pow(d->cr_ref, d->omega) * mean_rel;
    d->mft_free = 1.0 / (p->n_free * rate);
    const double mean_speed = std::sqrt(8.0 * k * p->t_free / (PI_D * m));
    d->mfp_free = mean_speed * d->mft_free;
    d->kn_free = d->mfp_free / p->box_height;
    d->sc_max = 9.0 * d->sigma_ref * std::sqrt(k * p->t_free / m); // Collision.cpp:23
    return DSMC_OK;
}

// WallModelName(), src/Boundary.cpp:15-24
const char *dsmc_wall_model_name(int wall_model)
{
    switch (wall_model) {
    case DSMC_WALL_SPECULAR: return "specular";
    case DSMC_WALL_DIFFUSE: return "diffuse";
    case DSMC_WALL_CLL: return "cll";
    }
    return nullptr;
}

const char *dsmc_status_string(int status)
{
    switch (status) {
    case DSMC_OK: return "ok";
    case DSMC_ERR_ARGUMENT: return "invalid argument";
    case DSMC_ERR_OUT_OF_DOMAIN: return "particle outside global domain";
    case DSMC_ERR_CELL_OVERFLOW: return "too many particles in cell";
    case DSMC_ERR_EXCHANGE: return "particle outside physical domain";
    case DSMC_ERR_CAPACITY: return "particle array capacity exceeded";
    case DSMC_ERR_BAD_CLL: return "CLL accommodation coefficients must be in [0, 1]";
    case DSMC_ERR_CUDA: return "CUDA runtime error";
    case DSMC_ERR_NO_DEVICE: return "no CUDA device";
    case DSMC_ERR_TIMEOUT: return "device-side wait timed out";
    case DSMC_ERR_STATE: return "call out of order";
    case DSMC_ERR_UNSUPPORTED: return "unsupported";
    case DSMC_ERR_TOO_LARGE: return "input larger than the fixed maximum of this entry point";
    }
    return "unknown status";
}

// The drag block of RunSimulation (src/Simulation.cpp:210-237, commented out
// in the reference): mean force over DragSamplingTime and the drag
// coefficient on the box's frontal area BoxHeight * DZ.
int dsmc_drag_report(const dsmc_params *p, const dsmc_derived *d, const dsmc_counters *c,
                     dsmc_drag *out)
{
    if (p == nullptr || d == nullptr || c == nullptr || out == nullptr)
        return DSMC_ERR_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->sampling_time = c->drag_sampling_time;
    out->rho_free = p->n_free * d->molecule_mass;
    out->area_ref = p->box_height * p->dz;
    out->box_collisions = c->drag_collision_count;
    out->box_collisions_window = c->drag_collision_count_window;
    if (!(c->drag_sampling_time > 0.0))
        return DSMC_ERR_STATE;
    const double q = 0.5 * out->rho_free * d->u_free * d->u_free * out->area_ref;
    out->mean_force_total = c->drag_impulse_total / c->drag_sampling_time;
    out->cd_total = out->mean_force_total / q;
    out->mean_force = c->drag_impulse_window / c->drag_sampling_time;
    out->cd = out->mean_force / q;
    return DSMC_OK;
}

// Printing(), src/Sampling.cpp:36-268: the Tecplot-style field and its JSON
// metadata, byte for byte in the reference's format.
int dsmc_write_field(const dsmc_params *p, const dsmc_derived *d, int64_t sample_step,
                     const dsmc_cell *cells, const char *results_dir)
{
    if (p == nullptr || d == nullptr || cells == nullptr || results_dir == nullptr)
        return DSMC_ERR_ARGUMENT;
    const char *wall = dsmc_wall_model_name(p->wall_model);
    if (wall == nullptr)
        return DSMC_ERR_ARGUMENT;
    const std::filesystem::path dir = std::filesystem::path(results_dir) / wall;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec)
        return DSMC_ERR_ARGUMENT;
    const auto field_path = dir / "DSMC2D_Field.plt";
    FILE *f = std::fopen(field_path.string().c_str(), "wt");
    if (f == nullptr)
        return DSMC_ERR_ARGUMENT;
    std::fprintf(f, "VARIABLES = \"X\" \"Y\" \"N\" \"Ux\" \"Uy\" \"Tx\" \"Ty\" \"T\"\n");
    std::fprintf(f, "ZONE I=%d J=%d\n", p->nx, p->ny);
    for (int k = 0; k < p->nx; k++) {
        for (int l = 0; l < p->ny; l++) {
            const dsmc_cell &c = cells[static_cast<int64_t>(k) * p->ny + l];
            const double x = p->x1 + (k + 0.5) * d->dx;
            const double y = p->y1 + (l + 0.5) * d->dy;
            double n = 0.0;
            double u[3] = {0.0, 0.0, 0.0};
            double txyz[3] = {0.0, 0.0, 0.0};
            if (sample_step > 0)
                n = d->weight * c.count_np / static_cast<int>(sample_step) / d->dv;
            if (c.count_np > 0.0) {
                for (int m = 0; m < 3; m++) {
                    u[m] = c.count_v[m] / c.count_np;
                    txyz[m] = d->molecule_mass * (c.count_vv[m][m] / c.count_np - u[m] * u[m]) /
                              K_BOLTZMANN;
                }
            }
            const double t = (txyz[0] + txyz[1] + txyz[2]) / 3.0;
            std::fprintf(f,
                         "%18.10e %18.10e %18.10e %18.10e %18.10e %18.10e %18.10e %18.10e\n",
                         x, y, n, u[0], u[1], txyz[0], txyz[1], t);
        }
    }
    const bool failed = std::ferror(f) != 0;
    if (std::fclose(f) != 0 || failed)
        return DSMC_ERR_ARGUMENT;

    std::ofstream meta(dir / "DSMC2D_Field.json");
    meta << std::setprecision(17) << "{\n  \"obstacle\": {\"type\": \"box\", \"center\": ["
         << p->box_x << ", " << p->box_y << "], \"width\": " << p->box_width
         << ", \"height\": " << p->box_height << "},\n"
         << "  \"angle_of_attack_degrees\": " << p->attack_angle << ",\n"
         << "  \"wall_model\": \"" << wall << "\",\n"
         << "  \"freestream\": {\"number_density\": " << p->n_free
         << ", \"temperature\": " << p->t_free << ", \"mach\": " << p->ma_free
         << ", \"molar_mass\": " << p->molar_mass << "},\n"
         << "  \"grid\": {\"nx\": " << p->nx << ", \"ny\": " << p->ny << ", \"bounds\": ["
         << p->x1 << ", " << p->x2 << ", " << p->y1 << ", " << p->y2
         << "], \"thickness\": " << p->dz << "},\n"
         << "  \"sampling\": {\"dt\": " << p->dt << ", \"steps\": " << p->n_step
         << ", \"first_step\": " << p->first_sampling_step << ", \"period\": "
         << p->sampling_period << ", \"particles_per_cell\": " << p->npc_free << "},\n"
         << "  \"collision_model\": {\"reference_diameter\": " << p->d_ref
         << ", \"viscosity_index\": " << p->viscosity_index
         << ", \"reference_temperature\": " << p->t_ref << "},\n"
         << "  \"wall_temperature\": " << p->t_wall;
    if (p->wall_model == DSMC_WALL_CLL)
        meta << ",\n  \"cll_accommodation\": {\"normal\": " << p->cll_normal
             << ", \"tangential\": " << p->cll_tangential << "}";
    meta << "\n}\n";
    meta.close();
    if (!meta)
        return DSMC_ERR_ARGUMENT;
    return DSMC_OK;
}

} // extern "C"
