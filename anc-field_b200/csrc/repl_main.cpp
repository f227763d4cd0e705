// anc-field: the interactive command loop of the reference executable
// (anc-field/src/main.cpp:32-143, anc-field/src/commandline.hpp:112-196)
// over the C ABI of include/afd.h. Same commands, argument types, error
// lines and progress output on stdout; diagnostics go to stderr so that
// stdout carries only the protocol that anc_field_py/ancfield.py parses.
//
// Additions, all optional and before `sd`/`sdt` (they set the parameters of
// the next simulation): `mode ref|fixed`, `dx <m>`, `c <m/s>`, `dt <s>`,
// `fs <Hz>`, `pmlfaces <mask>`, `graphs 0|1`, `precision fp32|fp16` (FP16
// field storage, with `mode fixed`). `vis` is headless: it records
// the y level and captures that plane on the device after every third step
// of a run (as the reference feeds its MJPEG stream); `visdump <file>`
// writes the plane of the latest field as text rows, or, for a file name
// ending in .npy, every captured frame as a float32 [frames][nz][nx] array.
#include <unistd.h>

#include <cerrno>
#include <climits>
#include <iterator>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/afd.h"
#include "model.hpp"

namespace {

bool parse_int(const std::string& t, int* out) {
    if (t.empty()) return false;
    errno = 0;
    char* end = nullptr;
    long v = std::strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != '\0' || errno == ERANGE || v < INT_MIN || v > INT_MAX) return false;
    *out = (int)v;
    return true;
}

bool parse_float(const std::string& t, float* out) {
    if (t.empty()) return false;
    errno = 0;
    char* end = nullptr;
    float v = std::strtof(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0' || errno == ERANGE) return false;
    *out = v;
    return true;
}

std::vector<std::string> split_list(const std::string& tok) {
    std::string s;
    for (char c : tok)
        if (c != '[' && c != ']') s += c;
    std::vector<std::string> parts;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) parts.push_back(item);
    return parts;
}

// Commandline::ToIntList / ToFloatList (commandline.hpp:57-105)
bool parse_int_list(const std::string& t, std::vector<int>* out) {
    out->clear();
    for (auto& p : split_list(t)) {
        int v;
        if (!parse_int(p, &v)) return false;
        out->push_back(v);
    }
    return true;
}

bool parse_float_list(const std::string& t, std::vector<float>* out) {
    out->clear();
    for (auto& p : split_list(t)) {
        float v;
        if (!parse_float(p, &v)) return false;
        out->push_back(v);
    }
    return true;
}

std::string self_dir() {
    char buf[4096];
    ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (n <= 0) return ".";
    buf[n] = '\0';
    std::string p(buf);
    size_t k = p.find_last_of('/');
    return k == std::string::npos ? "." : p.substr(0, k);
}

struct Repl {
    afd_params prm;
    afd_sim* sim = nullptr;
    std::vector<int> devices;
    uint32_t pml_faces = 63u;
    int vis_level = -1;
    using Handler = std::function<void(const std::vector<std::string>&)>;
    std::unordered_map<std::string, std::pair<Handler, std::vector<std::string>>> cmds;

    Repl() { afd_default_params(&prm); }
    ~Repl() {
        if (sim) afd_destroy(sim);
    }

    void fail_status(int st) {
        if (st != AFD_OK) std::cout << "Error: " << afd_last_error(sim) << "\n";
    }
    bool need_sim() {
        if (sim) return true;
        std::cout << "Error: no active simulation, select a device with sd or sdt first\n";
        return false;
    }
    void new_sim(int device) {
        if (sim) {
            afd_destroy(sim);
            sim = nullptr;
        }
        afd_params p = prm;
        p.device = device;
        int st = afd_create(&sim, &p);
        if (st != AFD_OK) {
            std::cout << "Error: " << afd_last_error(nullptr) << "\n";
            sim = nullptr;
        }
    }
    std::string device_name(int i) {
        char buf[256];
        if (afd_device_name(i, buf, sizeof buf) != AFD_OK) return std::string();
        return buf;
    }

    void add(const std::string& name, std::vector<std::string> types, Handler h) {
        cmds[name] = std::make_pair(std::move(h), std::move(types));
    }

    void setup() {
        add("lsd", {}, [this](const std::vector<std::string>&) {
            std::cout << "Available compute devices" << std::endl;
            for (int i = 0;; ++i) {
                std::string n = device_name(i);
                if (n.empty()) break;
                std::cout << i << ". " << n << std::endl;
            }
        });
        add("sd", {"int_list"}, [this](const std::vector<std::string>& a) {
            std::vector<int> ix;
            parse_int_list(a[0], &ix);
            for (int i : ix) {
                std::string n = device_name(i);
                if (n.empty()) {
                    std::cout << "Error: no compute device " << i << "\n";
                    return;
                }
                devices.push_back(i);
                std::cout << n << " added to active devices\n";
            }
            if (!devices.empty()) new_sim(devices[0]);
        });
        add("sdt", {"string"}, [this](const std::vector<std::string>& a) {
            if (a[0] != "cpu" && a[0] != "gpu") {
                std::cout << "Valid command arguments are 'cpu' or 'gpu'\n";
                return;
            }
            // Both kinds run on the first CUDA device: this build has no CPU path.
            std::string n = device_name(0);
            if (n.empty()) {
                std::cout << "Error: no CUDA device available\n";
                return;
            }
            devices.push_back(0);
            std::cout << n << " added to active devices\n";
            new_sim(0);
        });
        add("cd", {}, [this](const std::vector<std::string>&) {
            std::cout << "Compute devices removed\n";
            devices.clear();
        });
        add("load", {"file"}, [this](const std::vector<std::string>& a) {
            if (need_sim()) fail_status(afd_load(sim, a[0].c_str()));
        });
        add("addsource", {"float_list", "file"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            std::vector<float> pos;
            parse_float_list(a[0], &pos);
            if (pos.size() != 3) {
                std::cout << "Error: a position has three coordinates\n";
                return;
            }
            std::vector<float> sig;
            try {
                sig = afd::load_text_matrix(a[1], nullptr, nullptr);
            } catch (const std::exception& e) {
                std::cout << "Error: " << e.what() << "\n";
                return;
            }
            afd_info info;
            afd_get_info(sim, &info);
            // all sources of a run share one length (simulation.hpp:313-315)
            if (info.n_sources > 0 && (int64_t)sig.size() != src_len) {
                std::cout << "Error: all sources must have the same number of samples ("
                          << src_len << ")\n";
                return;
            }
            src_len = (int64_t)sig.size();
            fail_status(afd_add_source(sim, 0, pos.data(), sig.data(), (int64_t)sig.size()));
        });
        add("addmic", {"float_list"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            std::vector<float> pos;
            parse_float_list(a[0], &pos);
            if (pos.size() != 3) {
                std::cout << "Error: a position has three coordinates\n";
                return;
            }
            fail_status(afd_add_receiver(sim, pos.data()));
        });
        add("vis", {"float"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            float level;
            parse_float(a[0], &level);
            vis_level = (int)(level / prm.dx);
            // simulation.hpp:393-400 copies this plane after every third step
            // of a run; here into a ring of 64 device frames
            int st = afd_set_capture(sim, 0, 1, vis_level, 3, 64);
            if (st != AFD_OK) return fail_status(st);
            std::cerr << "vis: headless, plane y=" << vis_level << " captured every 3 steps on the device\n";
        });
        add("visdump", {"string"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            if (vis_level < 0) {
                std::cout << "Error: no vis level set\n";
                return;
            }
            afd_info info;
            afd_get_info(sim, &info);
            const std::string& path = a[0];
            if (path.size() > 4 && path.compare(path.size() - 4, 4, ".npy") == 0) {
                // every captured frame, oldest first: float32 [frames][nz][nx]
                std::vector<float> frames((size_t)64 * info.nx * info.nz);
                int32_t n = 0;
                int st = afd_get_frames(sim, frames.data(), (int64_t)frames.size(), nullptr, 0, &n);
                if (st != AFD_OK) return fail_status(st);
                if (!write_npy(path, frames.data(), n, info.nz, info.nx)) std::cout << "Error: cannot write " << path << "\n";
                return;
            }
            std::vector<float> plane((size_t)info.nx * info.nz);
            int st = afd_get_plane(sim, 0, 1, vis_level, plane.data(), (int64_t)plane.size());
            if (st != AFD_OK) return fail_status(st);
            try {
                afd::save_rows(a[0], plane.data(), info.nz, info.nx);
            } catch (const std::exception& e) {
                std::cout << "Error: " << e.what() << "\n";
            }
        });
        add("run", {"float"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            float sec;
            parse_float(a[0], &sec);
            // main.cpp:118-122: (int)(seconds * (real)fs)
            const float prod = sec * prm.fs;
            if (!(prod >= 0.0f && prod < 2147483648.0f)) {
                std::cout << "Error: run length out of range\n";
                return;
            }
            const int steps = (int)prod;
            int st = afd_run(sim, steps, &Repl::progress, nullptr);
            if (st != AFD_OK) fail_status(st);
        });
        add("save", {"string"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            afd_info info;
            afd_get_info(sim, &info);
            if (info.n_receivers == 0) {
                std::cout << "Error: no microphones to save\n";
                return;
            }
            std::vector<float> rec((size_t)(info.n_receivers * info.steps_done));
            int st = afd_get_receivers(sim, 0, rec.data(), (int64_t)rec.size());
            if (st != AFD_OK) return fail_status(st);
            try {
                afd::save_rows(a[0], rec.data(), info.n_receivers, info.steps_done);
            } catch (const std::exception& e) {
                std::cout << "Error: " << e.what() << "\n";
            }
        });
        add("minsize", {"float_list"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            std::vector<float> v;
            parse_float_list(a[0], &v);
            if (v.size() != 3) {
                std::cout << "Error: minsize takes three lengths\n";
                return;
            }
            fail_status(afd_set_min_size(sim, v[0], v[1], v[2]));
        });
        add("pml", {"int"}, [this](const std::vector<std::string>& a) {
            if (!need_sim()) return;
            int w;
            parse_int(a[0], &w);
            // simulation.hpp:263: the profile sits next to the executable
            const std::string path = self_dir() + "/ksi_profile_32.dat";
            std::vector<float> prof;
            std::ifstream probe(path);
            if (probe) {
                try {
                    prof = afd::load_text_matrix(path, nullptr, nullptr);
                } catch (const std::exception& e) {
                    std::cout << "Error: " << e.what() << "\n";
                    return;
                }
            } else {
                std::cerr << "pml: " << path << " not found, damping profile is zero\n";
            }
            if (prm.mode == AFD_MODE_REF || pml_faces == 63u) {
                fail_status(afd_set_pml_profile(sim, w, prof.data(), (int32_t)prof.size()));
            } else {
                afd_info info;
                afd_get_info(sim, &info);
                std::vector<float> k[3] = {std::vector<float>((size_t)info.nx, 0.0f),
                                           std::vector<float>((size_t)info.ny, 0.0f),
                                           std::vector<float>((size_t)info.nz, 0.0f)};
                const int n[3] = {info.nx, info.ny, info.nz};
                const int L = (int)prof.size();
                for (int ax = 0; ax < 3; ++ax)
                    for (int i = 0; i < L && i < n[ax]; ++i) {
                        if (pml_faces & (1u << (2 * ax))) k[ax][(size_t)i] = prof[(size_t)(L - 1 - i)];
                        if (pml_faces & (2u << (2 * ax))) k[ax][(size_t)(n[ax] - 1 - i)] = prof[(size_t)(L - 1 - i)];
                    }
                fail_status(afd_set_pml(sim, w, pml_faces, k[0].data(), k[1].data(), k[2].data()));
            }
        });
        // ---- additions ----
        add("mode", {"string"}, [this](const std::vector<std::string>& a) {
            if (a[0] == "ref") prm.mode = AFD_MODE_REF;
            else if (a[0] == "fixed") prm.mode = AFD_MODE_FIXED;
            else std::cout << "Valid command arguments are 'ref' or 'fixed'\n";
        });
        add("dx", {"float"}, [this](const std::vector<std::string>& a) { parse_float(a[0], &prm.dx); });
        add("c", {"float"}, [this](const std::vector<std::string>& a) { parse_float(a[0], &prm.c); });
        add("dt", {"float"}, [this](const std::vector<std::string>& a) { parse_float(a[0], &prm.dt); });
        add("fs", {"float"}, [this](const std::vector<std::string>& a) { parse_float(a[0], &prm.fs); });
        add("precision", {"string"}, [this](const std::vector<std::string>& a) {
            if (a[0] == "fp32") prm.storage = AFD_STORE_FP32;
            else if (a[0] == "fp16") prm.storage = AFD_STORE_FP16;
            else std::cout << "Valid command arguments are 'fp32' or 'fp16'\n";
        });
        add("graphs", {"int"}, [this](const std::vector<std::string>& a) {
            int v = 1;
            parse_int(a[0], &v);
            prm.graphs = v;
        });
        add("pmlfaces", {"int"}, [this](const std::vector<std::string>& a) {
            int v = 63;
            parse_int(a[0], &v);
            pml_faces = (uint32_t)v & 63u;
        });
    }

    // NumPy .npy (format 1.0) of a float32 [n][rows][cols] array.
    static bool write_npy(const std::string& path, const float* data, int64_t n, int64_t rows, int64_t cols) {
        std::string hdr = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(n) + ", " +
                          std::to_string(rows) + ", " + std::to_string(cols) + "), }";
        while ((10 + hdr.size() + 1) % 64) hdr += ' ';
        hdr += '\n';
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return false;
        const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
        const uint16_t len = (uint16_t)hdr.size();
        const unsigned char lenb[2] = {(unsigned char)(len & 0xff), (unsigned char)(len >> 8)};
        bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(lenb, 1, 2, f) == 2 &&
                  std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() &&
                  std::fwrite(data, sizeof(float), (size_t)(n * rows * cols), f) == (size_t)(n * rows * cols);
        ok = (std::fclose(f) == 0) && ok;
        return ok;
    }

    static int progress(int64_t i, int64_t steps, void*) {
        // simulation.hpp:403-409, 433
        if (i == 0 && steps > 0) std::cout << "BEGIN" << std::endl;
        std::cout << i << "/" << steps << std::endl;
        return 0;
    }

    int64_t src_len = 0;

    // Commandline::Run, commandline.hpp:112-196. End of input ends the loop.
    void loop(std::istream& in) {
        while (true) {
            std::cout << ">> " << std::flush;
            std::string line;
            if (!std::getline(in, line)) break;
            std::istringstream iss(line);
            std::vector<std::string> tok{std::istream_iterator<std::string>{iss},
                                         std::istream_iterator<std::string>{}};
            if (tok.empty()) continue;
            if (tok[0] == "quit") break;
            auto it = cmds.find(tok[0]);
            if (it == cmds.end()) {
                std::cout << "Error: unrecognized command\n";
                continue;
            }
            std::vector<std::string> args(tok.begin() + 1, tok.end());
            const auto& types = it->second.second;
            if (args.size() != types.size()) {
                std::cout << "Error: command " << tok[0] << " takes " << types.size() << " argument(s)\n";
                continue;
            }
            bool ok = true;
            for (size_t i = 0; i < args.size(); ++i) {
                const std::string& t = types[i];
                bool good = true;
                if (t == "int") {
                    int v;
                    good = parse_int(args[i], &v);
                } else if (t == "float") {
                    float v;
                    good = parse_float(args[i], &v);
                } else if (t == "file") {
                    if (!std::ifstream(args[i])) {
                        std::cout << "Error: file " << args[i] << " doesn't exist\n";
                        ok = false;
                        continue;
                    }
                } else if (t == "int_list") {
                    std::vector<int> v;
                    good = parse_int_list(args[i], &v);
                } else if (t == "float_list") {
                    std::vector<float> v;
                    good = parse_float_list(args[i], &v);
                }
                if (!good) {
                    std::cout << "Error: argument[" << i << "] should be a(n) " << t << "\n";
                    ok = false;
                }
            }
            if (ok) it->second.first(args);
            std::cout << std::flush;
        }
    }
};

}  // namespace

int main() {
    std::ios::sync_with_stdio(true);
    Repl r;
    r.setup();
    r.loop(std::cin);
    return EXIT_SUCCESS;
}
