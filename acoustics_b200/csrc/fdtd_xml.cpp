// fdtd_xml.cpp — a minimal XML attribute reader for the scene subset that
// ImpulseResponseParser consumes on this path (ImpulseResponseParser.cpp:55-751),
// plus the all_audio.dat writer (AudioOutput, AudioOutput.cpp:27-64).
//
// Accepted document:
//   <impulse_response>
//     <solver cellsize= timestepfrequency= [stop_time=] [number_of_timesteps=] [sound_speed=343]
//             [density=1.0] PML_width= PML_strength= [air_viscosity_alpha=0]
//             [boundary_condition_preset=0] [boundary_handling="rasterize"] [output_pattern=] .../>
//     <solver_control_policy type="static" gridresolution= [gridresolution_x|_y|_z=]
//             [domain_center_x|_y|_z=0]/>
//     <scene>
//       <analytic_sphere|analytic_box|analytic_ellipsoid center_x= center_y= center_z=
//             radius= | half_x= half_y= half_z= | semi_x= semi_y= semi_z=
//             [rotation="r00 r01 ... r22"] [acceleration="translation|pulsation" accel_amplitude=
//             accel_t0= accel_tau= accel_dir_x= ...] [velocity_x=.. gravity_x=..]/>
//       <constraint [direction=1] [sign=1] [height=0]/>
//     </scene>
//     <pressure_source>
//       <gaussian_pressure_source source_width_time= source_position_x= ... [source_width_space=]
//             [source_offset_time=0] [source_normalize_constant=] [source_sign_flip=0]/>
//     </pressure_source>
//     <listening_point_list><listening_point x= y= z=/></listening_point_list>
//   </impulse_response>
// Extensions beyond the reference schema: analytic primitives (instead of
// rigid_sound_object meshes), per-axis grid resolution, boundary acceleration
// and ballistic motion attributes.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

using fdtd::set_error;

namespace {

struct XNode {
    std::string name;
    std::map<std::string, std::string> attr;
    std::vector<std::unique_ptr<XNode>> kids;
    const XNode* child(const std::string& n) const {
        for (auto& k : kids)
            if (k->name == n) return k.get();
        return nullptr;
    }
};

struct XParser {
    const std::string& s;
    size_t i = 0;
    std::string err;
    explicit XParser(const std::string& str) : s(str) {}
    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    bool starts(const char* p) const { return s.compare(i, std::strlen(p), p) == 0; }
    bool skip_misc() {
        for (;;) {
            ws();
            if (starts("<?")) {
                size_t e = s.find("?>", i);
                if (e == std::string::npos) return false;
                i = e + 2;
            } else if (starts("<!--")) {
                size_t e = s.find("-->", i);
                if (e == std::string::npos) return false;
                i = e + 3;
            } else if (starts("<!")) {
                size_t e = s.find('>', i);
                if (e == std::string::npos) return false;
                i = e + 1;
            } else {
                return true;
            }
        }
    }
    std::unique_ptr<XNode> element() {
        if (!skip_misc() || i >= s.size() || s[i] != '<') { err = "expected '<'"; return nullptr; }
        ++i;
        auto n = std::make_unique<XNode>();
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/') n->name += s[i++];
        if (n->name.empty()) { err = "empty element name"; return nullptr; }
        for (;;) {
            ws();
            if (i >= s.size()) { err = "unterminated element <" + n->name + ">"; return nullptr; }
            if (s[i] == '/') {
                if (i + 1 < s.size() && s[i + 1] == '>') { i += 2; return n; }
                err = "bad '/' in <" + n->name + ">";
                return nullptr;
            }
            if (s[i] == '>') { ++i; break; }
            std::string key;
            while (i < s.size() && s[i] != '=' && !std::isspace((unsigned char)s[i])) key += s[i++];
            ws();
            if (i >= s.size() || s[i] != '=') { err = "attribute '" + key + "' without value"; return nullptr; }
            ++i;
            ws();
            if (i >= s.size() || (s[i] != '"' && s[i] != '\'')) { err = "attribute '" + key + "' not quoted"; return nullptr; }
            const char q = s[i++];
            size_t e = s.find(q, i);
            if (e == std::string::npos) { err = "unterminated attribute '" + key + "'"; return nullptr; }
            n->attr[key] = s.substr(i, e - i);
            i = e + 1;
        }
        // children until </name>
        for (;;) {
            // skip text
            while (i < s.size() && s[i] != '<') ++i;
            if (i >= s.size()) { err = "missing </" + n->name + ">"; return nullptr; }
            if (starts("<!--") || starts("<?") || starts("<!")) {
                if (!skip_misc()) { err = "unterminated comment"; return nullptr; }
                continue;
            }
            if (starts("</")) {
                size_t e = s.find('>', i);
                if (e == std::string::npos) { err = "unterminated close tag"; return nullptr; }
                std::string nm = s.substr(i + 2, e - i - 2);
                while (!nm.empty() && std::isspace((unsigned char)nm.back())) nm.pop_back();
                if (nm != n->name) { err = "mismatched </" + nm + "> for <" + n->name + ">"; return nullptr; }
                i = e + 1;
                return n;
            }
            auto k = element();
            if (!k) return nullptr;
            n->kids.push_back(std::move(k));
        }
    }
};

bool get_real(const XNode* n, const char* key, double& v, bool required, double dflt, std::string& err) {
    auto it = n->attr.find(key);
    if (it == n->attr.end()) {
        if (required) { err = std::string("missing required attribute '") + key + "' of <" + n->name + ">"; return false; }
        v = dflt;
        return true;
    }
    char* end = nullptr;
    v = std::strtod(it->second.c_str(), &end);
    if (end == it->second.c_str()) { err = std::string("attribute '") + key + "' is not a number"; return false; }
    return true;
}

}  // namespace

struct fdtd_scene {
    fdtd_scene_desc desc{};
    std::vector<fdtd_object_desc> objects;
    std::vector<fdtd_plane_desc> planes;
    std::vector<fdtd_gaussian_source_desc> sources;
    std::vector<double> listeners;
    std::vector<fdtd_mesh_desc> meshes;
    std::vector<std::vector<double>> mverts;
    std::vector<std::vector<int32_t>> mtris;
    std::vector<fdtd_keyframe_track> tracks;
    std::vector<std::vector<double>> tframes;
    int32_t steps = 0;
    std::string output_pattern;
};

extern "C" {

fdtd_status fdtd_scene_from_xml(const char* path, fdtd_scene** out) {
    if (!path || !out) return (set_error(nullptr, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    *out = nullptr;
    std::ifstream f(path, std::ios::binary);
    if (!f) return (set_error(nullptr, std::string("cannot open ") + path), FDTD_ERR_IO);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    XParser xp(text);
    auto root = xp.element();
    if (!root) return (set_error(nullptr, "XML: " + xp.err), FDTD_ERR_INVALID_ARG);
    if (root->name != "impulse_response") return (set_error(nullptr, "root element must be <impulse_response>"), FDTD_ERR_INVALID_ARG);
    std::unique_ptr<fdtd_scene> sc(new fdtd_scene());
    std::string err;
    // features outside this path are named before any file they refer to is read
    if (const XNode* scene = root->child("scene"))
        for (auto& kid : scene->kids) {
            const XNode* n = kid.get();
            if (n->name == "acoustic_shaders")
                return (set_error(nullptr, "<acoustic_shaders> (modal transfer shaders) is not on this path"),
                        FDTD_ERR_UNSUPPORTED);
            if (n->name == "rigid_object_sequence" || n->name == "shell_object")
                return (set_error(nullptr, "<" + n->name + "> (object-file sequences, shell objects) is not on this path"),
                        FDTD_ERR_UNSUPPORTED);
            if (n->name == "rigid_sound_object") {
                auto on = [&](const char* a) {
                    auto it = n->attr.find(a);
                    return it != n->attr.end() && std::atof(it->second.c_str()) != 0.0;
                };
                if (on("has_modal_source") || n->attr.count("add_shader_by_id") || n->attr.count("mode_file") ||
                    on("has_acc_noise_source"))
                    return (set_error(nullptr, "<rigid_sound_object> with modal vibration sources or shaders is not on "
                                               "this path (a <rigid_object> mesh is)"),
                            FDTD_ERR_UNSUPPORTED);
            }
            if (n->name == "rigid_object" &&
                (n->attr.count("has_harmonic_source") || n->attr.count("speaker_file") || n->attr.count("has_speaker_shader")))
                return (set_error(nullptr, "<rigid_object> speaker / harmonic vibration sources are not on this path"),
                        FDTD_ERR_UNSUPPORTED);
        }
    const XNode* solver = root->child("solver");
    if (!solver) return (set_error(nullptr, "missing <solver>"), FDTD_ERR_INVALID_ARG);
    {
        auto tp = solver->attr.find("time_parallel");
        if (tp != solver->attr.end() && std::atof(tp->second.c_str()) != 0.0)
            return (set_error(nullptr, "time-parallel chunking (time_parallel) is not on this path"), FDTD_ERR_UNSUPPORTED);
    }
    fdtd_scene_desc& D = sc->desc;
    double freq = 0, v = 0;
    // GetSolverSettings (ImpulseResponseParser.cpp:493-575)
    bool ok = get_real(solver, "sound_speed", D.sound_speed, false, 343.0, err) &&
              get_real(solver, "density", D.density, false, 1.0, err) &&
              get_real(solver, "cellsize", D.cell_size, true, 0, err) &&
              get_real(solver, "timestepfrequency", freq, true, 0, err) &&
              get_real(solver, "stop_time", D.end_time, false, 0.0, err) &&
              get_real(solver, "PML_width", D.pml_width, true, 0, err) &&
              get_real(solver, "PML_strength", D.pml_strength, true, 0, err) &&
              get_real(solver, "air_viscosity_alpha", D.air_viscosity_alpha, false, 0.0, err) &&
              get_real(solver, "number_of_timesteps", v, false, 0.0, err);
    if (!ok) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
    sc->steps = (int32_t)v;
    D.time_step = 1.0 / freq;
    if (!get_real(solver, "boundary_condition_preset", v, false, 0.0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
    D.boundary_condition_preset = (int32_t)v;
    // ImpulseResponseParser.cpp:547-555
    auto bh = solver->attr.find("boundary_handling");
    D.boundary_handling = FDTD_BOUNDARY_RASTERIZE;
    if (bh != solver->attr.end()) {
        if (bh->second == "fully_coupled") D.boundary_handling = FDTD_BOUNDARY_FULLY_COUPLED;
        else if (bh->second != "rasterize")
            return (set_error(nullptr, "boundary handling type not understood: " + bh->second), FDTD_ERR_INVALID_ARG);
    }
    auto op = solver->attr.find("output_pattern");
    sc->output_pattern = op == solver->attr.end() ? std::string("%s") : op->second;
    // solver_control_policy, static (ImpulseResponseParser.cpp:615-627) + per-axis extension
    const XNode* pol = root->child("solver_control_policy");
    if (!pol) return (set_error(nullptr, "missing <solver_control_policy>"), FDTD_ERR_INVALID_ARG);
    auto ty = pol->attr.find("type");
    if (ty == pol->attr.end() || ty->second != "static")
        return (set_error(nullptr, "only the static solver_control_policy is on this path"), FDTD_ERR_UNSUPPORTED);
    double g = 0;
    if (!get_real(pol, "gridresolution", g, false, 0.0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
    const char* axes[3] = {"gridresolution_x", "gridresolution_y", "gridresolution_z"};
    const char* cen[3] = {"domain_center_x", "domain_center_y", "domain_center_z"};
    for (int d = 0; d < 3; ++d) {
        double gd = 0;
        if (!get_real(pol, axes[d], gd, false, g, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
        if (!(gd > 0)) return (set_error(nullptr, "gridresolution missing"), FDTD_ERR_INVALID_ARG);
        D.divisions[d] = (int32_t)gd;
        if (!get_real(pol, cen[d], D.domain_center[d], false, 0.0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
    }
    // scene objects
    if (const XNode* scene = root->child("scene")) {
        for (auto& kid : scene->kids) {
            const XNode* n = kid.get();
            const bool mesh_obj = n->name == "rigid_object" || n->name == "rigid_sound_object";
            if (mesh_obj || n->name == "analytic_sphere" || n->name == "analytic_box" || n->name == "analytic_ellipsoid") {
                fdtd_object_desc o{};
                o.shape = mesh_obj ? FDTD_SHAPE_MESH
                                   : n->name == "analytic_sphere" ? FDTD_SHAPE_SPHERE
                                   : n->name == "analytic_box"    ? FDTD_SHAPE_BOX
                                                                  : FDTD_SHAPE_ELLIPSOID;
                const char* c3[3] = {"center_x", "center_y", "center_z"};
                const char* ip3[3] = {"initial_position_x", "initial_position_y", "initial_position_z"};
                for (int d = 0; d < 3; ++d)
                    if (!get_real(n, mesh_obj ? ip3[d] : c3[d], o.center[d], false, 0.0, err))
                        return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                if (mesh_obj) {
                    // ImpulseResponseParser.cpp:210-219: <working_directory>/<object_prefix>.obj,
                    // scaled (the distance-field resolution has no counterpart: distances are exact)
                    auto wd = n->attr.find("working_directory"), op = n->attr.find("object_prefix");
                    if (wd == n->attr.end() || op == n->attr.end())
                        return (set_error(nullptr, "<" + n->name + "> needs working_directory and object_prefix"),
                                FDTD_ERR_INVALID_ARG);
                    double scale = 1.0;
                    if (!get_real(n, "scale", scale, false, 1.0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                    std::string file = wd->second + "/" + op->second + ".obj";
                    if (!std::ifstream(file) && !file.empty() && file[0] != '/') {
                        // relative to the XML file when not found from the working directory
                        const std::string xp_dir = std::string(path).substr(0, std::string(path).find_last_of('/') + 1);
                        if (std::ifstream(xp_dir + file)) file = xp_dir + file;
                    }
                    std::vector<double> v;
                    std::vector<int32_t> t;
                    if (!fdtd::read_obj(file.c_str(), scale, v, t, err)) return (set_error(nullptr, err), FDTD_ERR_IO);
                    o.mesh = (int32_t)sc->meshes.size();
                    sc->meshes.push_back(fdtd_mesh_desc{(int32_t)(v.size() / 3), (int32_t)(t.size() / 3), nullptr, nullptr});
                    sc->mverts.push_back(std::move(v));
                    sc->mtris.push_back(std::move(t));
                } else if (o.shape == FDTD_SHAPE_SPHERE) {
                    if (!get_real(n, "radius", o.size[0], true, 0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                } else {
                    const char* pre = o.shape == FDTD_SHAPE_BOX ? "half_" : "semi_";
                    const char* ax = "xyz";
                    for (int d = 0; d < 3; ++d) {
                        std::string key = std::string(pre) + ax[d];
                        if (!get_real(n, key.c_str(), o.size[d], true, 0, err)) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                    }
                }
                for (int i = 0; i < 9; ++i) o.rotation[i] = (i % 4 == 0) ? 1.0 : 0.0;
                auto rot = n->attr.find("rotation");
                if (rot != n->attr.end()) {
                    std::istringstream rs(rot->second);
                    for (int i = 0; i < 9; ++i)
                        if (!(rs >> o.rotation[i])) return (set_error(nullptr, "rotation needs 9 numbers"), FDTD_ERR_INVALID_ARG);
                }
                auto acc = n->attr.find("acceleration");
                if (acc != n->attr.end()) {
                    if (acc->second == "translation") o.accel_kind = FDTD_ACCEL_GAUSSIAN_TRANSLATION;
                    else if (acc->second == "pulsation") o.accel_kind = FDTD_ACCEL_GAUSSIAN_PULSATION;
                    else if (acc->second != "none") return (set_error(nullptr, "unknown acceleration kind"), FDTD_ERR_INVALID_ARG);
                    const char* ad[3] = {"accel_dir_x", "accel_dir_y", "accel_dir_z"};
                    ok = get_real(n, "accel_amplitude", o.accel_amplitude, o.accel_kind != 0, 0, err) &&
                         get_real(n, "accel_t0", o.accel_t0, false, 0.0, err) &&
                         get_real(n, "accel_tau", o.accel_tau, o.accel_kind != 0, 1.0, err);
                    for (int d = 0; d < 3 && ok; ++d) ok = get_real(n, ad[d], o.accel_dir[d], false, d == 2 ? 1.0 : 0.0, err);
                    if (!ok) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                }
                const char* vk[3] = {"velocity_x", "velocity_y", "velocity_z"};
                const char* gk[3] = {"gravity_x", "gravity_y", "gravity_z"};
                for (int d = 0; d < 3; ++d) {
                    if (n->attr.count(vk[d]) || n->attr.count(gk[d])) o.motion = FDTD_MOTION_BALLISTIC;
                    if (!get_real(n, vk[d], o.velocity[d], false, 0.0, err) || !get_real(n, gk[d], o.gravity[d], false, 0.0, err))
                        return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                }
                // keyframes (ImpulseResponseParser.cpp:250-264): file_kinematics= kinematics_frame_rate=
                auto kin = n->attr.find("file_kinematics");
                if (kin != n->attr.end() && kin->second != "N/A") {
                    double rate = 0;
                    if (!get_real(n, "kinematics_frame_rate", rate, true, 0, err) || !(rate > 0))
                        return (set_error(nullptr, err.empty() ? "kinematics_frame_rate must be positive" : err),
                                FDTD_ERR_INVALID_ARG);
                    std::string kf = kin->second;
                    if (!std::ifstream(kf) && !kf.empty() && kf[0] != '/') {
                        const std::string xp_dir = std::string(path).substr(0, std::string(path).find_last_of('/') + 1);
                        if (std::ifstream(xp_dir + kf)) kf = xp_dir + kf;
                    }
                    std::vector<double> frames;
                    if (!fdtd::read_kinematics(kf.c_str(), frames, err)) return (set_error(nullptr, err), FDTD_ERR_IO);
                    o.motion = FDTD_MOTION_KEYFRAMED;
                    sc->tracks.push_back(fdtd_keyframe_track{(int32_t)sc->objects.size(), (int32_t)(frames.size() / 7),
                                                             1.0 / rate, nullptr});
                    sc->tframes.push_back(std::move(frames));
                }
                sc->objects.push_back(o);
            } else if (n->name == "constraint") {
                // ImpulseResponseParser.cpp:433-449
                fdtd_plane_desc p{};
                double dir = 1, sign = 1;
                if (!get_real(n, "direction", dir, false, 1.0, err) || !get_real(n, "sign", sign, false, 1.0, err) ||
                    !get_real(n, "height", p.height, false, 0.0, err))
                    return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
                p.normal_dir = (int32_t)dir;
                p.normal_sign = (int32_t)sign;
                sc->planes.push_back(p);
            } else if (n->name == "rigid_object_sequence" || n->name == "shell_object") {
                return (set_error(nullptr, "<" + n->name + "> (keyframed object sequences, shell objects) is not on this path"),
                        FDTD_ERR_UNSUPPORTED);
            }
        }
    }
    // pressure sources (GetPressureSources, ImpulseResponseParser.cpp:647-675)
    if (const XNode* ps = root->child("pressure_source")) {
        for (auto& kid : ps->kids) {
            const XNode* n = kid.get();
            if (n->name != "gaussian_pressure_source") continue;
            fdtd_gaussian_source_desc g2{};
            double flip = 0;
            ok = get_real(n, "source_width_time", g2.width_time, true, 0, err) &&
                 get_real(n, "source_width_space", g2.width_space, false, D.sound_speed * g2.width_time, err) &&
                 get_real(n, "source_offset_time", g2.offset_time, false, 0.0, err) &&
                 get_real(n, "source_sign_flip", flip, false, 0.0, err) &&
                 get_real(n, "source_position_x", g2.position[0], true, 0, err) &&
                 get_real(n, "source_position_y", g2.position[1], true, 0, err) &&
                 get_real(n, "source_position_z", g2.position[2], true, 0, err);
            if (!ok) return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
            const double scaleSign = flip > 1E-10 ? -1.0 : 1.0;
            double nc = 0;
            if (!get_real(n, "source_normalize_constant", nc, false,
                          1.0 / std::pow(std::sqrt(2.0 * M_PI) * g2.width_space, 3), err))
                return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
            g2.normalize_constant = nc * scaleSign;
            sc->sources.push_back(g2);
        }
    }
    // listeners (GetListeningPoints, ImpulseResponseParser.cpp:677-703)
    if (const XNode* ll = root->child("listening_point_list")) {
        for (auto& kid : ll->kids) {
            const XNode* n = kid.get();
            if (n->name != "listening_point") continue;
            double p[3];
            if (!get_real(n, "x", p[0], true, 0, err) || !get_real(n, "y", p[1], true, 0, err) || !get_real(n, "z", p[2], true, 0, err))
                return (set_error(nullptr, err), FDTD_ERR_INVALID_ARG);
            sc->listeners.insert(sc->listeners.end(), p, p + 3);
        }
    }
    D.n_objects = (int32_t)sc->objects.size();
    D.n_constraints = (int32_t)sc->planes.size();
    D.n_sources = (int32_t)sc->sources.size();
    D.n_listeners = (int32_t)(sc->listeners.size() / 3);
    D.objects = sc->objects.data();
    D.constraints = sc->planes.data();
    D.sources = sc->sources.data();
    D.listeners = sc->listeners.data();
    for (size_t m = 0; m < sc->meshes.size(); ++m) {
        sc->meshes[m].vertices = sc->mverts[m].data();
        sc->meshes[m].triangles = sc->mtris[m].data();
    }
    D.n_meshes = (int32_t)sc->meshes.size();
    D.meshes = sc->meshes.empty() ? nullptr : sc->meshes.data();
    for (size_t k = 0; k < sc->tracks.size(); ++k) sc->tracks[k].frames = sc->tframes[k].data();
    D.n_tracks = (int32_t)sc->tracks.size();
    D.tracks = sc->tracks.empty() ? nullptr : sc->tracks.data();
    *out = sc.release();
    return FDTD_OK;
}

const fdtd_scene_desc* fdtd_scene_desc_get(const fdtd_scene* sc) { return sc ? &sc->desc : nullptr; }
int32_t fdtd_scene_number_of_steps(const fdtd_scene* sc) { return sc ? sc->steps : 0; }
const char* fdtd_scene_output_pattern(const fdtd_scene* sc) { return sc ? sc->output_pattern.c_str() : ""; }
void fdtd_scene_free(fdtd_scene* sc) { delete sc; }

// AudioOutput::WriteAndResetBuffer (AudioOutput.cpp:56-64): raw doubles, no header
fdtd_status fdtd_audio_append(const char* path, const double* data, int64_t count) {
    if (!path || (count > 0 && !data) || count < 0) return (set_error(nullptr, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    FILE* f = std::fopen(path, "ab");
    if (!f) return (set_error(nullptr, std::string("cannot open ") + path), FDTD_ERR_IO);
    const size_t w = std::fwrite(data, sizeof(double), (size_t)count, f);
    std::fclose(f);
    if (w != (size_t)count) return (set_error(nullptr, "short write"), FDTD_ERR_IO);
    return FDTD_OK;
}

}  // extern "C"
