// What the reference's engine/factory.cuh becomes after the maintainer's edit
// that INTEGRATION.md describes: the rule-packing format it defines
// (PackedTrees, pack_trees; engine/factory.cuh:20-40) stays, and the
// FactoryContext struct with its kernels (:42-217) is replaced by the B200
// library's drop-in class.  The reference's drivers include "factory.cuh" (or
// "../engine/factory.cuh"); compiled with this directory ahead of the
// reference's engine/ directory (and -I-, so a quoted include does not look
// beside the including file first), they get this file and the rest of the
// reference's headers unchanged.  Test infrastructure: tests/test_dropin.py
// builds the reference's verify/verify_cuda.cu and engine/gp_engine.cu this
// way, as plain C++ linked against libsidr_b200.so.
#pragma once
#include <cstdint>
#include <vector>

#include "sim_core.hpp"
#include "sim_host.hpp"
#include "vocab.hpp"

// The flat rule format the evaluator takes: post-order opcodes, two
// arguments per node, and each rule's offset and length.
struct PackedTrees {
    std::vector<int32_t> ops, args;
    std::vector<int32_t> offsets, lengths;
};

inline PackedTrees pack_trees(const std::vector<NodeP>& trees) {
    PackedTrees out;
    for (const NodeP& t : trees) {
        const Compiled c = compile_rmod(t);
        out.offsets.push_back((int32_t)out.ops.size());
        out.lengths.push_back((int32_t)c.ops.size());
        out.ops.insert(out.ops.end(), c.ops.begin(), c.ops.end());
        for (const auto& a : c.args) {
            out.args.push_back(a[0]);
            out.args.push_back(a[1]);
        }
    }
    return out;
}

#include "sidr_factory.hpp"
using FactoryContext = sidr::FactoryContextT<SimData, PackedTrees>;
