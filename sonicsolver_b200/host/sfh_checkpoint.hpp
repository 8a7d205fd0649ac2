// sfh_checkpoint.hpp -- restart files of `sfg_run`.
//
// The document follows the reference's field checkpoint (CheckpointIO::write
// -> FieldIO::write with restart fields only,
// src/infrastructure/io/checkpoint/SF_checkpoint.h:5 and
// src/infrastructure/io/field/SF_field.cpp:67-79): a JSON mapping
// {"formatVersion": 1, "fields": {name: {"descriptor": {...}, "size": N,
// "values": [...]}}} with the conserved variables as its restart fields --
// rho (scalar), rhoU (vector) and rhoE (scalar), one entry per node, values
// written with 17 significant digits so that they read back to the last
// bit.  Beside "fields" it carries the run's clock, which the reference
// takes from the case instead: "time", "steps", "nextOutput" (the next
// output time) and "outputs" (output files written so far), so that a run
// restarted from it takes the dt sequence of the run that wrote it.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace sfh {

struct Checkpoint {
    int nodes[3] = {1, 1, 1};
    double time = 0.0;
    int64_t steps = 0;
    double next_output = 0.0;  // +inf: no output schedule
    int outputs = 0;
    std::vector<double> q;     // conserved AoS [k][j][i][v] over the nodes
};

// Writes the document; returns false when the file cannot be written or a
// value is not finite (the reference refuses non-finite checkpoints).
bool write_checkpoint(const std::string& path, const Checkpoint& c);

// Reads a document written by write_checkpoint (or any JSON document of that
// shape).  Throws std::runtime_error naming the file and the problem.
Checkpoint read_checkpoint(const std::string& path);

}  // namespace sfh
