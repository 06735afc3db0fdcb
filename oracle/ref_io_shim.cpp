/*
 * ORACLE PIN — test infrastructure, not product code.
 *
 * The reference's own output and restart code, compiled for the host from the reference tree
 * where it lies (this shim and the two reference sources below are compiled together by
 * oracle/Makefile; nothing is copied):
 *   WbWriterVtkXmlBinary  src/basics/writer/WbWriterVtkXmlBinary.cpp  (writeOctsWithNodeData :1306,
 *                         writeParallelFile :141, writeCollectionForTimeSeries :88)
 *   BinaryRestartObject   src/gpu/core/Restart/RestartObject.cpp      (serialize_internal,
 *                         deserialize_internal)
 * into _ref/libvfref_io64.so (real = double) and _ref/libvfref_io32.so (real = float). The tests
 * write the same data through this shim and through virtualfluids_b200.output and compare the
 * files byte for byte.
 *
 * RestartObject.cpp also holds serialize()/deserialize(), which read a Parameter; the shim never
 * calls them and fills the public `fs` member instead. The four Parameter members they name are
 * defined below only so that the library links; they abort if they are ever reached.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <basics/writer/WbWriterVtkXmlBinary.h>

#include "Parameter/Parameter.h"
#include "Restart/RestartObject.h"

std::shared_ptr<LBMSimulationParameter> Parameter::getParH(int) const { std::abort(); }
int Parameter::getFine() const { std::abort(); }
int Parameter::getCoarse() const { std::abort(); }
int Parameter::getD3Qxx() { std::abort(); }

namespace
{
int copy_name(const std::string &s, char *out, int out_len)
{
    if (!out || out_len <= 0)
        return (int)s.size();
    std::strncpy(out, s.c_str(), (size_t)out_len - 1);
    out[out_len - 1] = '\0';
    return (int)s.size();
}
} // namespace

extern "C" {

int refio_real_bytes() { return (int)sizeof(real); }

/* WbWriterVtkXmlBinary::writeOctsWithNodeData: xyz[3 n_nodes] (x, y, z per node), cells[8 n_cells] in
   the tuple order of UbTupleUInt8 (1..8), data[n_data * n_nodes] one row per name. The written
   file's name goes to out_name. */
int refio_write_octs(const char *filename, int n_nodes, const float *xyz, int n_cells, const int *cells, int n_data,
                     const char *const *names, const double *data, char *out_name, int out_len)
{
    std::vector<UbTupleFloat3> nodes((size_t)n_nodes);
    for (int i = 0; i < n_nodes; ++i)
        nodes[(size_t)i] = makeUbTuple(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    std::vector<UbTupleUInt8> octs((size_t)n_cells);
    for (int c = 0; c < n_cells; ++c) {
        const int *o = cells + 8 * (size_t)c;
        octs[(size_t)c] = makeUbTuple((unsigned int)o[0], (unsigned int)o[1], (unsigned int)o[2], (unsigned int)o[3],
                                      (unsigned int)o[4], (unsigned int)o[5], (unsigned int)o[6], (unsigned int)o[7]);
    }
    std::vector<std::string> datanames;
    std::vector<std::vector<double>> nodedata;
    for (int s = 0; s < n_data; ++s) {
        datanames.emplace_back(names[s]);
        nodedata.emplace_back(data + (size_t)s * n_nodes, data + (size_t)(s + 1) * n_nodes);
    }
    const std::string written = WbWriterVtkXmlBinary::getInstance()->writeOctsWithNodeData(filename, nodes, octs,
                                                                                          datanames, nodedata);
    return copy_name(written, out_name, out_len);
}

/* WbWriterVtkXmlBinary::writeParallelFile (no cell data, as FileWriter::writeCollectionFile) */
int refio_write_parallel_file(const char *filename, int n_pieces, const char *const *pieces, int n_names,
                              const char *const *names, char *out_name, int out_len)
{
    std::vector<std::string> src(pieces, pieces + n_pieces), point(names, names + n_names), cell;
    return copy_name(WbWriterVtkXmlBinary::getInstance()->writeParallelFile(filename, src, point, cell), out_name,
                     out_len);
}

/* WbWriterVtkXmlBinary::writeCollectionForTimeSeries: n_steps time steps, counts[i] files each,
   the file names of all steps one after the other */
int refio_write_time_series(const char *filename, int n_steps, const unsigned *timesteps, const int *counts,
                            const char *const *files, int separate_groups, char *out_name, int out_len)
{
    std::map<uint, std::vector<std::string>> series;
    int k = 0;
    for (int i = 0; i < n_steps; ++i)
        for (int j = 0; j < counts[i]; ++j)
            series[timesteps[i]].emplace_back(files[k++]);
    return copy_name(WbWriterVtkXmlBinary::getInstance()->writeCollectionForTimeSeries(filename, series,
                                                                                       separate_groups != 0),
                     out_name, out_len);
}

/* BinaryRestartObject::serialize_internal of n_levels arrays of `real` (sizes[i] values each) */
int refio_restart_write(const char *filename, int n_levels, const int64_t *sizes, const real *const *arrays)
{
    std::unique_ptr<RestartObject> r(new BinaryRestartObject());
    for (int i = 0; i < n_levels; ++i)
        r->fs.emplace_back(arrays[i], arrays[i] + sizes[i]);
    r->serialize_internal(filename);
    return 0;
}

/* BinaryRestartObject::deserialize_internal: the number of levels, then (when sizes / arrays are
   given) each level's size and values (arrays[i] holds room for max_values values) */
int refio_restart_read(const char *filename, int max_levels, int64_t *sizes, real *const *arrays, int64_t max_values)
{
    std::unique_ptr<RestartObject> r(new BinaryRestartObject());
    r->deserialize_internal(filename);
    const int n = (int)r->fs.size();
    for (int i = 0; i < n && i < max_levels; ++i) {
        if (sizes)
            sizes[i] = (int64_t)r->fs[(size_t)i].size();
        if (arrays && arrays[i] && (int64_t)r->fs[(size_t)i].size() <= max_values)
            std::memcpy(arrays[i], r->fs[(size_t)i].data(), r->fs[(size_t)i].size() * sizeof(real));
    }
    return n;
}

} // extern "C"
