// GPU_Runner: the reference simulator's runner interface
// (Simulator::circuitRunner, src/simulator.hpp:85-97) implemented over
// libquokka_gpu.so, for the runner_type=GPU slot the reference leaves as a
// stub (src/simulator.cpp:225-228, :253-256).
//
// It takes the gate objects the reference's own MEM parser builds
// (Simulator::setGate_MEM, src/simulator.cpp:542-597), turns each into a
// qk_gate and hands the list to the engine; the state lives in HBM
// (qk_sv) from construction to destruction.  Errors follow the reference's
// convention: a message on cerr and exit(1).
#pragma once

#include <string>
#include <vector>

#include "quokka_gpu.h"
#include "simulator.hpp"

class GPU_Runner : public Simulator::circuitRunner {
public:
    // MEM_Runner::MEM_Runner (src/MEM_Runner.cpp:57-88): a 2^seg.N state in
    // |0...0> (or read from the engine's init_file key).  The .ini is read
    // again for the engine's own keys (precision, fuse_width, dump_format,
    // init_file), which the reference ignores.
    explicit GPU_Runner(const std::string &ini);
    // Writes the dump the .ini asks for (after Simulator::run's timed span:
    // the reference's text dump, src/simulator.cpp:696-704, or with
    // dump_format=bin the raw complex128 state), then frees the device state.
    ~GPU_Runner() override;
    // MEM_Runner::run(std::vector<Gate*>&) (src/MEM_Runner.cpp:101-134):
    // per-gate kernels, or fused passes when fuse_width > 0.
    void run(std::vector<Gate *> &circuit) override;
    // MEM_Runner::run(std::vector<std::vector<Gate*>>&) (src/MEM_Runner.cpp:
    // 136-185): the groups' gates as one fused plan, VSWAPs as renamings.
    void run(std::vector<std::vector<Gate *>> &subcircuits) override;

    qk_sv *state() const { return sv; }
    // One gate object of the reference's MEM parser as a qk_gate record.
    static qk_gate to_qk(const Gate *g);

private:
    qk_config cfg;
    qk_sv *sv = nullptr;
};
