// outputs.hpp -- the reference's output files: the run directory written by make_context
// (grid_spacing.txt, coordinate_mapping.txt, mesh_info.json; src/params.hpp:296-505) and the
// detectors of register_default_detectors (src/params.hpp:681-790): MeshDetector,
// FieldMovie2D and PointFieldDetector (src/detectors/*.hpp), same names, layout and text.
//
// With gain, the two-level detectors main() creates (src/3D_FDTD_version008.cpp:174-198,
// src/two_level_detectors.hpp): populations/ (first and last Nu/Ng frames, inversion_time.csv,
// metadata_populations.json), polarization/polarization_time.csv and tls_global_history.csv.
// (TLSGlobalHistory's plotting script is not written: it is not an output format.)
//
// This part is host-only: the plan (which files, which slices), the text files and the
// writer thread.  The stepper captures movie slices and probe samples on the device and
// hands them to an OutputWriter (solver.cu).
#pragma once

#include "setup.hpp"

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace fdtd {

struct MeshDetectorPlan {  // MeshDetectorConfig + MeshDetector::initialize (mesh_detector.hpp:10-95)
    std::string name;
    int plane = 0;  // 0 XY (z = const), 1 XZ, 2 YZ
    std::size_t index = 0;
    real coord = 0;  // cell centre of the slice, physical coordinates
    bool mesh_lines = true, spacing = true;
};

struct MoviePlan {  // FieldMovie2DConfig + FieldMovie2D::initialize (field_movie_2d.hpp:11-100)
    std::string name, pattern;
    int component = 2, plane = 0;
    std::size_t index = 0;
    real coord = 0;
    // Slice extent as the reference writes it: XY (NxT, NyT), XZ (NxT, NzT), YZ (NyT, NzT);
    // value (a, b) at offset a * dim2 + b.
    std::size_t dim1 = 0, dim2 = 0;
};

struct PointPlan {  // PointFieldDetector::initialize (point_field_detector.hpp:41-105)
    std::string name;
    std::size_t i = 0, j = 0, k = 0;
    std::vector<int> components;
    real px = 0, py = 0, pz = 0;
};

struct OutputPlan {
    std::string run_tag = "3D_FDTD_v008_output";  // RUN_TAG
    bool float64 = true;                           // WRITE_FLOAT64
    std::vector<MeshDetectorPlan> meshes;
    std::vector<MoviePlan> movies;
    std::vector<PointPlan> points;
    bool tls = false;  // the setup has gain: write the two-level detectors' files
    // PolarizationDiagnostics' cell: PROBE_X/Y/Z mapped like main() does (no clamp);
    // mon_valid is false when that cell lies outside the field grid.
    bool mon_valid = false;
    std::size_t mon_i = 0, mon_j = 0, mon_k = 0;
    // what the end-of-run metadata needs
    std::size_t NxT = 0, NyT = 0, NzT = 0, save_every = 1, n_steps = 0;
    double dt = 0;
};

// One line of each two-level CSV at step n (the record() functions of
// PopulationTimeSeriesDetector, PolarizationDiagnostics and TLSGlobalHistory).
std::string inversion_line(uint64_t n, double dt, double total_Nu, double total_Ng);
std::string polarization_line(uint64_t n, double dt, double Pz_center, double dPz_dt_center, double P_energy);
std::string global_history_line(uint64_t n, double dt, double Nu_total, double Ng_total);
// PopulationTimeSeriesDetector::finalize's metadata_populations.json.
void write_population_metadata(const OutputPlan& plan, const std::string& root);

// Reads RUN_TAG, WRITE_FLOAT64, MESH_DETECTORS and FIELD_MOVIE_2D_DETECTORS from the
// setup's parameter file and takes the point detectors from the setup.  Throws
// std::runtime_error on a malformed entry or frame pattern.
OutputPlan make_output_plan(const SimSetup& S);

// <root>/frames/<run_tag>
std::string run_dir(const OutputPlan& plan, const std::string& root);

// Writes every file the reference writes before its time loop: the three run files, the
// mesh detectors' files, the movies' and point detectors' metadata.json, and empty
// <component>_ts.bin files.  Throws std::runtime_error when a file cannot be written.
void write_setup_outputs(const SimSetup& S, const OutputPlan& plan, const std::string& root);

// Frame file of movie m: snprintf(pattern, frame) in the movie's directory.
std::string frame_path(const OutputPlan& plan, const std::string& root, std::size_t m, uint64_t frame);

// Component name used in file names (field_component_name, idetector.hpp:31-50).
const char* component_name(int c);

// One background thread that writes files in submission order.  A job first runs its
// wait function (the stepper passes a wait on the copy that fills the buffer), then writes
// (append or truncate) the bytes, then runs its done function (which frees the buffer).
class OutputWriter {
public:
    struct Job {
        std::function<void()> wait, done;
        std::function<std::string()> text;  // when set: the bytes to write, made after wait()
        std::string path;
        const void* data = nullptr;
        std::size_t bytes = 0;
        bool append = false;
    };
    OutputWriter();
    ~OutputWriter();
    void submit(Job j);
    // Blocks until every submitted job has finished; rethrows the first write error.
    void drain();

private:
    void loop();
    std::mutex mu_;
    std::condition_variable cv_, idle_;
    std::deque<Job> q_;
    bool stop_ = false, busy_ = false;
    std::string error_;
    std::thread th_;
};

}  // namespace fdtd
