// `next` -- the command-line driver, with the reference's contract
// (src/begrun.cpp:40-137, argparse/argparse.cpp:21-61):
//
//   next <input.txt> <threads> <dt> <dump_interval> <vtk|vtu|hdf5>
//
// Each loop iteration takes dt = computeAdaptiveDt(bodies, dt_arg), runs one
// KDK step, advances the simulation time and writes dump_<k>.<fmt> whenever
// the time passes the next dump time; typing `q` (or `Q`) ends the run.  The
// bodies stay on the GPU between steps and are copied back only for dumps;
// a dump's file is written by a host thread while the GPU runs the next
// steps (the writer of one dump is waited for before the next copy back).
//
// Additions, all optional and off by default so the contract is unchanged:
//   NEXT_MAX_STEPS / NEXT_T_END  stop after that many steps / that time
//   NEXT_PHYSICS, NEXT_PRECISION, NEXT_THETA, NEXT_EPS, NEXT_LEAF_CAP,
//   NEXT_DEVICE                  see gravity/engine.h
// `threads` only sizes host-side work (the gravity path runs on the GPU).
// HDF5 is accepted as a format name but this build has no libhdf5, so the
// run stops with an error before the first step.
#include <poll.h>
#include <unistd.h>

#include <cstdlib>
#include <future>
#include <iostream>
#include <string>

#include "gravity/engine.h"
#include "io/load_particle.hpp"
#include "io/vtk_save.h"
#include "io/vtu_save.h"

namespace {

enum class Format { VTK, VTU, HDF5 };

bool quit_requested() {
    pollfd pfd{0, POLLIN, 0};
    if (poll(&pfd, 1, 0) <= 0 || !(pfd.revents & POLLIN)) return false;
    char c = 0;
    if (read(0, &c, 1) != 1) return false;
    return c == 'q' || c == 'Q';
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 6) {
        std::cerr << "Usage: next <input.txt> <threads> <dt> <dump_interval> <vtk|vtu|hdf5>\n";
        return 1;
    }
    const std::string input = argv[1];
    int threads = 0;
    double dt_arg = 0, dump_interval = 0;
    try {
        threads = std::stoi(argv[2]);
        dt_arg = std::stod(argv[3]);
        dump_interval = std::stod(argv[4]);
    } catch (const std::exception&) {
        std::cerr << "Usage: next <input.txt> <threads> <dt> <dump_interval> <vtk|vtu|hdf5>\n";
        return 1;
    }
    const std::string fmt = argv[5];
    Format format;
    if (fmt == "vtk") format = Format::VTK;
    else if (fmt == "vtu") format = Format::VTU;
    else if (fmt == "hdf5") format = Format::HDF5;
    else {
        std::cerr << "Choose a file format: vtk, vtu, or hdf5\n";
        return 1;
    }
    if (format == Format::HDF5) {
        std::cerr << "hdf5 output is not available in this build (no libhdf5); use vtk or vtu\n";
        return 1;
    }
    const long max_steps = std::getenv("NEXT_MAX_STEPS") ? std::atol(std::getenv("NEXT_MAX_STEPS")) : -1;
    const double t_end = std::getenv("NEXT_T_END") ? std::atof(std::getenv("NEXT_T_END")) : -1.0;

    std::cout << "\n _  _ ________   _________ \n| \\ | |  ____\\ \\ / /__   __|\n|  \\| | |__   \\ V /   | |   \n"
                 "| . ` |  __|   > <    | |   \n| |\\  | |____ / . \\   | |   \n|_| \\_|______/_/ \\_\\  |_|   \n"
              << std::endl;
    std::cout << " Threads:   " << threads << std::endl;
    std::cout << " Precision: FP64" << std::endl;

    Particle particles = LoadParticlesFromFile(input);
    std::cout << " Particles: " << particles.size() << std::endl;
    if (particles.size() == 0) return 0;

    try {
        next_gpu::Engine& eng = next_gpu::engine();
        eng.upload(particles);
        double sim_time = 0, next_dump = 0;
        long dumps = 0, steps = 0;
        std::future<void> writer;   // the previous dump's file, being written
        for (;;) {
            const double dt = eng.adaptive_dt(dt_arg);
            eng.step(dt);
            sim_time += dt;
            ++steps;
            if (sim_time >= next_dump) {
                if (writer.valid()) writer.get();   // `particles` is free again
                eng.download(particles);
                std::string out = "dump_" + std::to_string(dumps) + (format == Format::VTK ? ".vtk" : ".vtu");
                // only dumps touch `particles` (the state lives on the GPU), so the
                // file can be written while the next steps run
                writer = std::async(std::launch::async, [&particles, out, format] {
                    if (format == Format::VTK) SaveVTK(particles, out);
                    else SaveVTU(particles, out);
                });
                std::cout << "[Dump " << dumps << "] t = " << sim_time << ", file: " << out << std::endl;
                next_dump += dump_interval;
                ++dumps;
            }
            if (quit_requested()) {
                std::cout << "Exiting..." << std::endl;
                break;
            }
            if ((max_steps >= 0 && steps >= max_steps) || (t_end >= 0 && sim_time >= t_end)) break;
        }
        if (writer.valid()) writer.get();
    } catch (const std::exception& e) {
        std::cerr << "next: " << e.what() << std::endl;
        return 2;
    }
    return 0;
}
