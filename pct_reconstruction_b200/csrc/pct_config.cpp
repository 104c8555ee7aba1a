// pct_config.cpp -- runtime configuration with the reference's parameter names.
//
// The reference fixes its parameters as macros in B.h:333-480 (the built program) and, in the
// unbuilt variant, reads settings.cfg through Configurations.h:838-987 ("KEY = value // comment"
// lines, typed setters, then set_dependent_parameters).  Here every parameter is a runtime field
// of pct_config; derived values are computed by pct_config_finalize with the same expressions
// as the B.h macros (so that, e.g., COLUMNS = int(2*R / VOXEL_WIDTH) rounds identically).
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <cmath>
#include <string>

#include "../../include/pct_api.h"

extern "C" size_t pct_config_size(void) { return sizeof(pct_config); }

extern "C" void pct_config_default(pct_config* c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    // Grid (B.h:378-393); zero means "derive in pct_config_finalize".
    c->VOXEL_WIDTH = 0.0625;
    c->VOXEL_HEIGHT = 0.0625;
    c->VOXEL_THICKNESS = 0.25;
    c->RECON_CYL_RADIUS = 8.0;
    // Tracker / binning (B.h:344-367)
    c->GANTRY_ANGLE_INTERVAL = 4.0;
    c->SSD_T_SIZE = 35.0;
    c->SSD_V_SIZE = 9.0;
    c->T_BIN_SIZE = 0.0625;
    c->V_BIN_SIZE = 0.25;
    c->ANGULAR_BIN_SIZE = 3.0;
    c->SIGMAS_TO_KEEP = 2;
    c->SAMPLE_STD_DEV = 1;
    // FBP (B.h:162, 368-371, 474-480, 743-745)
    c->SINOGRAM_FILTER = PCT_SHEPP_LOGAN;
    c->MEDIAN_FILTER_FBP = 1;
    c->FBP_MED_FILTER_RADIUS = 3;
    c->SOURCE_RADIUS = 260.7;
    c->FBP_THRESHOLD = 0.6;
    c->RSP_AIR = 0.00113;
    // Hulls (B.h:395-405, 170, 228-230)
    c->SC_LOWER_THRESHOLD = 0.0;
    c->SC_UPPER_THRESHOLD = 0.0;
    c->MSC_LOWER_THRESHOLD = -10.0;
    c->MSC_UPPER_THRESHOLD = 0.0;
    c->MSC_DIFF_THRESH = 150;
    c->SM_LOWER_THRESHOLD = 6.0;
    c->SM_UPPER_THRESHOLD = 21.0;
    c->SM_SCALE_THRESHOLD = 1.0;
    c->ENDPOINTS_HULL = PCT_MSC_HULL;
    c->SC_ON = 0;
    c->MSC_ON = 1;
    c->SM_ON = 0;
    // MLP (B.h:409-411): MLP_U_STEP = VOXEL_WIDTH/2 derived when 0
    c->MIN_MLP_LENGTH = 30;
    // DROP (B.h:335, 419-423)
    c->LAMBDA = 0.0001f;
    c->DROP_BLOCK_SIZE = 204800;
    c->ITERATIONS = 10;
    c->HISTORIES_PER_BLOCK = 640;
    c->PRECISION = PCT_PRECISION_EXACT;
    c->SCATTER_MODE = PCT_SCATTER_ATOMIC;
    c->THREADS_PER_HISTORY = 0;
    c->PATH_CHUNK_BLOCKS = 16;
    c->EXACT_FAST_POINTS = 1;
    c->PATH_CTA_THREADS = 128;
    c->PATH_ORDER_WINDOW = 0;
    // Reader (B.h:291, 302, 355-357)
    c->DATA_IN_MM = 1;
    c->USE_CONT_ANGLES = 0;
    // TVS (B.h:427-443)
    c->TVS_ON = 1;
    c->TVS_OLD = 0;
    c->TVS_FIRST = 1;
    c->TVS_CONDITIONED = 1;
    c->TVS_REPETITIONS = 5;
    c->TVS_L_0 = 0;
    c->TVS_A = 0.5;
    c->TVS_MIN_ETA = 1e-40;
    c->TV_THRESHOLD = 0.0;
    c->TVS_SEED = 0x5eed;
    // Projection algorithm, ordering, air threshold (B.h:175, 181, 416-419, 464-465)
    c->PROJECTION_ALGORITHM = PCT_DROP;
    c->PSI_SIGN = 1;
    c->ETA = 2.5;
    c->RECON_HISTORY_ORDERING = PCT_SEQUENTIAL;
    c->IDENTIFY_X_N_AIR = 0;
    c->PRIME_OFFSET = 26410633;
    c->X_N_AIR_THRESHOLD = 0.1;
    // S-curve attenuation (B.h:178, 467-470)
    c->S_CURVE_ON = 0;
    c->S_CURVE = PCT_SIGMOID;
    c->DUAL_SIDED_S_CURVE = 1;
    c->SIGMOID_MID_SHIFT = 10;
    c->SIGMOID_STEEPNESS = 1.25;
}

namespace {

enum FieldType { F_INT, F_DOUBLE, F_FLOAT, F_INT64 };

struct FieldDesc {
    const char* name;
    FieldType type;
    size_t offset;
};

#define FD_I(n) {#n, F_INT, offsetof(pct_config, n)}
#define FD_D(n) {#n, F_DOUBLE, offsetof(pct_config, n)}
#define FD_F(n) {#n, F_FLOAT, offsetof(pct_config, n)}
#define FD_L(n) {#n, F_INT64, offsetof(pct_config, n)}

const FieldDesc kFields[] = {
    FD_I(COLUMNS), FD_I(ROWS), FD_I(SLICES), FD_I(NUM_VOXELS),
    FD_D(VOXEL_WIDTH), FD_D(VOXEL_HEIGHT), FD_D(VOXEL_THICKNESS),
    FD_D(RECON_CYL_RADIUS), FD_D(RECON_CYL_HEIGHT),
    FD_D(GANTRY_ANGLE_INTERVAL), FD_D(SSD_T_SIZE), FD_D(SSD_V_SIZE),
    FD_D(T_BIN_SIZE), FD_D(V_BIN_SIZE), FD_D(ANGULAR_BIN_SIZE),
    FD_I(T_BINS), FD_I(V_BINS), FD_I(ANGULAR_BINS), FD_I(NUM_BINS),
    FD_I(SIGMAS_TO_KEEP), FD_I(SAMPLE_STD_DEV),
    FD_I(SINOGRAM_FILTER), FD_I(MEDIAN_FILTER_FBP), FD_I(FBP_MED_FILTER_RADIUS),
    FD_D(SOURCE_RADIUS), FD_D(FBP_THRESHOLD), FD_D(RSP_AIR),
    FD_D(SC_LOWER_THRESHOLD), FD_D(SC_UPPER_THRESHOLD), FD_D(MSC_LOWER_THRESHOLD),
    FD_D(MSC_UPPER_THRESHOLD), FD_D(SM_LOWER_THRESHOLD), FD_D(SM_UPPER_THRESHOLD),
    FD_D(SM_SCALE_THRESHOLD), FD_I(MSC_DIFF_THRESH), FD_I(ENDPOINTS_HULL),
    FD_I(SC_ON), FD_I(MSC_ON), FD_I(SM_ON),
    FD_D(MLP_U_STEP), FD_I(MIN_MLP_LENGTH),
    FD_F(LAMBDA), FD_I(DROP_BLOCK_SIZE), FD_I(ITERATIONS), FD_I(HISTORIES_PER_BLOCK),
    FD_I(PRECISION), FD_I(SCATTER_MODE), FD_I(THREADS_PER_HISTORY), FD_I(PATH_CHUNK_BLOCKS), FD_I(EXACT_FAST_POINTS), FD_I(PATH_CTA_THREADS), FD_I(PATH_ORDER_WINDOW),
    FD_I(DATA_IN_MM), FD_I(USE_CONT_ANGLES), FD_D(T_SHIFT), FD_D(U_SHIFT), FD_D(V_SHIFT),
    FD_I(TVS_ON), FD_I(TVS_OLD), FD_I(TVS_FIRST), FD_I(TVS_CONDITIONED), FD_I(TVS_REPETITIONS), FD_I(TVS_L_0),
    FD_D(TVS_A), FD_D(TVS_MIN_ETA), FD_D(TV_THRESHOLD), FD_L(TVS_SEED),
    FD_I(PROJECTION_ALGORITHM), FD_I(PSI_SIGN), FD_D(ETA), FD_I(RECON_HISTORY_ORDERING), FD_I(IDENTIFY_X_N_AIR),
    FD_L(PRIME_OFFSET), FD_D(X_N_AIR_THRESHOLD),
    FD_I(S_CURVE_ON), FD_I(S_CURVE), FD_I(DUAL_SIDED_S_CURVE), FD_I(SIGMOID_MID_SHIFT), FD_D(SIGMOID_STEEPNESS),
};

// settings.cfg spellings that differ from the B.h names (settings.cfg:21-60, Configurations.h).
struct Alias {
    const char* cfg_key;
    const char* field;
};
const Alias kAliases[] = {
    {"SIGMAS_2_KEEP", "SIGMAS_TO_KEEP"},
    {"SLICE_THICKNESS", "VOXEL_THICKNESS"},
    {"FBP_FILTER_TYPE", "SINOGRAM_FILTER"},
    {"HULL_TYPE", "ENDPOINTS_HULL"},
    {"A", "TVS_A"},
    {"L_0", "TVS_L_0"},
};

// Symbolic enum values accepted for the enum-valued keys.
struct EnumName {
    const char* name;
    int value;
};
const EnumName kEnumNames[] = {
    {"RAM_LAK", PCT_RAM_LAK}, {"SHEPP_LOGAN", PCT_SHEPP_LOGAN}, {"UNFILTERED", PCT_UNFILTERED},
    {"SC_HULL", PCT_SC_HULL}, {"MSC_HULL", PCT_MSC_HULL}, {"SM_HULL", PCT_SM_HULL},
    {"FBP_HULL", PCT_FBP_HULL}, {"EXACT", PCT_PRECISION_EXACT}, {"MIXED", PCT_PRECISION_MIXED},
    {"MIXED_COMPENSATED", PCT_PRECISION_MIXED_COMPENSATED},
    {"ATOMIC", PCT_SCATTER_ATOMIC}, {"DETERMINISTIC", PCT_SCATTER_DETERMINISTIC},
    {"DROP", PCT_DROP}, {"ROBUSTA", PCT_ROBUSTA}, {"ROBUSTB", PCT_ROBUSTB},
    {"SEQUENTIAL", PCT_SEQUENTIAL}, {"PRIME_PERMUTATION", PCT_PRIME_PERMUTATION},
    {"SIGMOID", PCT_SIGMOID}, {"TANH", PCT_TANH}, {"ATAN", PCT_ATAN}, {"ERF", PCT_ERF},
    {"LIN_OVER_ROOT", PCT_LIN_OVER_ROOT},
    {"true", 1}, {"false", 0}, {"ON", 1}, {"OFF", 0},
};

bool parse_int_value(const char* v, long* out)
{
    for (const EnumName& e : kEnumNames)
        if (strcasecmp(v, e.name) == 0) {
            *out = e.value;
            return true;
        }
    char* end = nullptr;
    double d = strtod(v, &end);
    if (end == v || *end != '\0') return false;
    if (d != std::floor(d) || std::fabs(d) > 2147483647.0) return false;
    *out = (long)d;
    return true;
}

}  // namespace

namespace {

// Reason of the calling thread's last pct_config_set / pct_config_load / pct_config_finalize failure.
thread_local std::string g_config_error;

pct_status config_fail(const std::string& why)
{
    g_config_error = why;
    return PCT_ERR_ARG;
}

}  // namespace

extern "C" pct_status pct_config_set(pct_config* c, const char* key, const char* value)
{
    if (!c || !key || !value) return config_fail("pct_config_set: null argument");
    const char* name = key;
    for (const Alias& a : kAliases)
        if (strcmp(key, a.cfg_key) == 0) name = a.field;
    for (const FieldDesc& f : kFields) {
        if (strcmp(name, f.name) != 0) continue;
        char* base = reinterpret_cast<char*>(c) + f.offset;
        if (f.type == F_INT) {
            long v;
            if (!parse_int_value(value, &v)) return config_fail(std::string(key) + ": not an integer or a known name: " + value);
            *reinterpret_cast<int32_t*>(base) = (int32_t)v;
        } else if (f.type == F_INT64) {
            char* end = nullptr;
            long long v = strtoll(value, &end, 0);
            if (end == value || *end != '\0') return config_fail(std::string(key) + ": not an integer: " + value);
            *reinterpret_cast<int64_t*>(base) = (int64_t)v;
        } else {
            char* end = nullptr;
            double d = strtod(value, &end);
            if (end == value || *end != '\0') return config_fail(std::string(key) + ": not a number: " + value);
            if (f.type == F_DOUBLE) *reinterpret_cast<double*>(base) = d;
            else *reinterpret_cast<float*>(base) = (float)d;
        }
        return PCT_OK;
    }
    return config_fail(std::string("unknown key ") + key);
}

extern "C" pct_status pct_config_load(pct_config* c, const char* path)
{
    if (!c || !path) return config_fail("pct_config_load: null argument");
    FILE* f = fopen(path, "r");
    if (!f) {
        g_config_error = std::string("cannot open ") + path;
        return PCT_ERR_IO;
    }
    char line[1024];
    pct_status st = PCT_OK;
    std::string first_error;
    while (fgets(line, sizeof(line), f)) {
        // strip "// comment"
        char* cm = strstr(line, "//");
        if (cm) *cm = '\0';
        char* eq = strchr(line, '=');
        if (!eq) continue;
        *eq = '\0';
        std::string k(line), v(eq + 1);
        auto trim = [](std::string& s) {
            size_t a = 0, b = s.size();
            while (a < b && isspace((unsigned char)s[a])) a++;
            while (b > a && isspace((unsigned char)s[b - 1])) b--;
            s = s.substr(a, b - a);
        };
        trim(k);
        trim(v);
        if (k.empty()) continue;
        if (v.size() >= 2 && v.front() == '"' && v.back() == '"') continue;  // paths and names
        pct_status s = pct_config_set(c, k.c_str(), v.c_str());
        // Keys of the reference's I/O, logging and host options have no engine counterpart
        // and are skipped; a known key with a malformed value is an error.
        if (s != PCT_OK) {
            bool known = false;
            for (const FieldDesc& fd : kFields) known |= strcmp(k.c_str(), fd.name) == 0;
            for (const Alias& a : kAliases) known |= strcmp(k.c_str(), a.cfg_key) == 0;
            if (known && st == PCT_OK) first_error = g_config_error;
            if (known) st = PCT_ERR_ARG;
        }
    }
    fclose(f);
    // the skipped keys of other subsystems leave their own messages; keep the first real error
    g_config_error = st == PCT_OK ? std::string() : std::string(path) + ": " + first_error;
    return st;
}

extern "C" const char* pct_config_last_error(void) { return g_config_error.c_str(); }

extern "C" pct_status pct_config_finalize(pct_config* c)
{
    if (!c) return config_fail("pct_config_finalize: null configuration");
    g_config_error.clear();
    if (c->VOXEL_WIDTH <= 0 || c->VOXEL_HEIGHT <= 0 || c->VOXEL_THICKNESS <= 0)
        return config_fail("VOXEL_WIDTH, VOXEL_HEIGHT and VOXEL_THICKNESS must be positive");
    if (c->RECON_CYL_RADIUS <= 0) return config_fail("RECON_CYL_RADIUS must be positive");
    // RECON_CYL_HEIGHT = (SSD_V_SIZE - 1.0) (B.h:376)
    if (c->RECON_CYL_HEIGHT <= 0) c->RECON_CYL_HEIGHT = (c->SSD_V_SIZE - 1.0);
    // COLUMNS = int(RECON_CYL_DIAMETER/VOXEL_WIDTH), ROWS likewise, SLICES = int(H/SLICE_THICKNESS)
    if (c->COLUMNS <= 0) c->COLUMNS = (int)((2 * c->RECON_CYL_RADIUS) / c->VOXEL_WIDTH);
    if (c->ROWS <= 0) c->ROWS = (int)((2 * c->RECON_CYL_RADIUS) / c->VOXEL_HEIGHT);
    if (c->SLICES <= 0) c->SLICES = (int)(c->RECON_CYL_HEIGHT / c->VOXEL_THICKNESS);
    if (c->COLUMNS <= 0 || c->ROWS <= 0 || c->SLICES <= 0)
        return config_fail("the grid has no voxels (COLUMNS, ROWS or SLICES derived as 0)");
    long long nv = (long long)c->COLUMNS * c->ROWS * c->SLICES;
    if (nv + (long long)c->COLUMNS * c->ROWS > 0x7fffffffLL)
        return config_fail("NUM_VOXELS plus one spare slice exceeds 2^31 - 1");
    c->NUM_VOXELS = (int32_t)nv;
    // T_BINS = int(SSD_T_SIZE / T_BIN_SIZE + 0.5) etc. (B.h:356-362)
    if (c->T_BIN_SIZE <= 0 || c->V_BIN_SIZE <= 0 || c->ANGULAR_BIN_SIZE <= 0)
        return config_fail("T_BIN_SIZE, V_BIN_SIZE and ANGULAR_BIN_SIZE must be positive");
    c->T_BINS = (int)(c->SSD_T_SIZE / c->T_BIN_SIZE + 0.5);
    c->V_BINS = (int)(c->SSD_V_SIZE / c->V_BIN_SIZE + 0.5);
    c->ANGULAR_BINS = (int)(360 / c->ANGULAR_BIN_SIZE + 0.5);
    long long nb = (long long)c->T_BINS * c->V_BINS * c->ANGULAR_BINS;
    if (nb <= 0 || nb > 0x7fffffffLL) return config_fail("NUM_BINS must lie in [1, 2^31 - 1]");
    c->NUM_BINS = (int32_t)nb;
    // MLP_U_STEP = VOXEL_WIDTH/2 (B.h:411)
    if (c->MLP_U_STEP <= 0) c->MLP_U_STEP = (c->VOXEL_WIDTH / 2);
    if (c->MLP_U_STEP < 0.00005) return config_fail("MLP_U_STEP is below the lookup tables' step of 0.00005 cm");
    if (c->DROP_BLOCK_SIZE <= 0 || c->ITERATIONS < 0 || c->HISTORIES_PER_BLOCK < 0)
        return config_fail("DROP_BLOCK_SIZE must be positive, ITERATIONS and HISTORIES_PER_BLOCK non-negative");
    if (c->PRECISION < PCT_PRECISION_EXACT || c->PRECISION > PCT_PRECISION_MIXED_COMPENSATED)
        return config_fail("PRECISION must be EXACT, MIXED or MIXED_COMPENSATED");
    if (c->SCATTER_MODE != PCT_SCATTER_ATOMIC && c->SCATTER_MODE != PCT_SCATTER_DETERMINISTIC)
        return config_fail("SCATTER_MODE must be ATOMIC or DETERMINISTIC");
    int tph = c->THREADS_PER_HISTORY;
    if (tph != 0 && tph != 32)  // the DROP-block kernel runs one warp per history
        return config_fail("THREADS_PER_HISTORY must be 0 or 32 (one warp per history)");
    if (c->TVS_REPETITIONS < 0 || c->TVS_L_0 < 0) return config_fail("TVS_REPETITIONS and L_0 must be non-negative");
    if (c->PATH_CHUNK_BLOCKS < 0) return config_fail("PATH_CHUNK_BLOCKS must be non-negative");
    if (c->EXACT_FAST_POINTS != 0 && c->EXACT_FAST_POINTS != 1) return config_fail("EXACT_FAST_POINTS must be 0 or 1");
    if (c->PATH_CTA_THREADS != 64 && c->PATH_CTA_THREADS != 128 && c->PATH_CTA_THREADS != 256)
        return config_fail("PATH_CTA_THREADS must be 64, 128 or 256");
    if (c->PATH_ORDER_WINDOW < 0 || c->PATH_ORDER_WINDOW > (1 << 24))
        return config_fail("PATH_ORDER_WINDOW must lie in [0, 2^24]");
    if (!(c->TVS_A > 0.0 && c->TVS_A < 1.0) || !(c->TVS_MIN_ETA > 0.0 && c->TVS_MIN_ETA < 1.0))
        return config_fail("A and TVS_MIN_ETA must lie in (0, 1)");
    if (c->PROJECTION_ALGORITHM != PCT_DROP && c->PROJECTION_ALGORITHM != PCT_ROBUSTA &&
        c->PROJECTION_ALGORITHM != PCT_ROBUSTB)
        return config_fail("PROJECTION_ALGORITHM must be DROP, ROBUSTA or ROBUSTB");
    if (c->PSI_SIGN != 1 && c->PSI_SIGN != -1) return config_fail("PSI_SIGN must be 1 or -1");
    if (c->RECON_HISTORY_ORDERING != PCT_SEQUENTIAL && c->RECON_HISTORY_ORDERING != PCT_PRIME_PERMUTATION)
        return config_fail("RECON_HISTORY_ORDERING must be SEQUENTIAL or PRIME_PERMUTATION");
    if (c->PRIME_OFFSET <= 0) return config_fail("PRIME_OFFSET must be positive");
    if (c->SCATTER_MODE == PCT_SCATTER_DETERMINISTIC && c->PROJECTION_ALGORITHM == PCT_ROBUSTB)
        return config_fail("SCATTER_MODE DETERMINISTIC is not built for PROJECTION_ALGORITHM ROBUSTB");
    if (c->S_CURVE_ON != 0 && c->S_CURVE_ON != 1) return config_fail("S_CURVE_ON must be 0 or 1");
    if (c->DUAL_SIDED_S_CURVE != 0 && c->DUAL_SIDED_S_CURVE != 1)
        return config_fail("DUAL_SIDED_S_CURVE must be 0 or 1");
    if (c->S_CURVE < PCT_SIGMOID || c->S_CURVE > PCT_LIN_OVER_ROOT)
        return config_fail("S_CURVE must be SIGMOID, TANH, ATAN, ERF or LIN_OVER_ROOT");
    if (!std::isfinite(c->SIGMOID_STEEPNESS)) return config_fail("SIGMOID_STEEPNESS must be finite");
    // The attenuation is built into the exact DROP update (the reference's only user of it).
    if (c->S_CURVE_ON && (c->PRECISION != PCT_PRECISION_EXACT || c->PROJECTION_ALGORITHM != PCT_DROP))
        return config_fail("S_CURVE_ON needs PRECISION EXACT and PROJECTION_ALGORITHM DROP");
    return PCT_OK;
}
