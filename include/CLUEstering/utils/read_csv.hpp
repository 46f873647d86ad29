// read_csv.hpp -- points from CSV files (reference: include/CLUEstering/utils/detail/read_csv.hpp:14-89).
// read_csv: one header line, then rows "x0,...,x{N-1},weight".  read_output: rows
// "x0,...,x{N-1},weight,cluster_id[,...]"; the points come back marked as clustered.
#pragma once

#include "CLUEstering/data_structures/Points.hpp"

#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace clue {

  namespace detail {
    inline std::vector<std::vector<std::string>> read_rows(const std::string& file_path) {
      std::ifstream file(file_path);
      if (!file.is_open()) throw std::runtime_error("Could not open file: " + file_path);
      std::vector<std::vector<std::string>> rows;
      std::string line;
      std::getline(file, line);  // header
      while (std::getline(file, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        std::vector<std::string> fields;
        std::stringstream ss(line);
        std::string f;
        while (std::getline(ss, f, ',')) fields.push_back(f);
        rows.push_back(std::move(fields));
      }
      return rows;
    }
  }  // namespace detail

  template <std::size_t NDim>
  inline PointsHost<NDim> read_csv(Dim<NDim> dim, const std::string& file_path) {
    const auto rows = detail::read_rows(file_path);
    PointsHost<NDim> points(dim, static_cast<int32_t>(rows.size()));
    for (std::size_t i = 0; i < rows.size(); ++i) {
      if (rows[i].size() < NDim + 1) throw std::runtime_error("Too few columns in " + file_path);
      for (std::size_t d = 0; d < NDim; ++d) points.coords(d)[i] = std::stof(rows[i][d]);
      points.weights()[i] = std::stof(rows[i][NDim]);
    }
    return points;
  }

  template <std::size_t NDim>
  inline PointsHost<NDim> read_output(Dim<NDim> dim, const std::string& file_path) {
    const auto rows = detail::read_rows(file_path);
    PointsHost<NDim> points(dim, static_cast<int32_t>(rows.size()));
    for (std::size_t i = 0; i < rows.size(); ++i) {
      if (rows[i].size() < NDim + 2) throw std::runtime_error("Too few columns in " + file_path);
      for (std::size_t d = 0; d < NDim; ++d) points.coords(d)[i] = std::stof(rows[i][d]);
      points.weights()[i] = std::stof(rows[i][NDim]);
      points.clusterIndexes()[i] = std::stoi(rows[i][NDim + 1]);
    }
    points.mark_clustered();
    return points;
  }

  // The queue-taking forms of the reference (utils/read_csv.hpp:17-30).
  template <std::size_t NDim, concepts::Queue TQueue>
  inline PointsHost<NDim> read_csv(TQueue&, const std::string& file_path) {
    return read_csv(Dim<NDim>{}, file_path);
  }
  template <std::size_t NDim, concepts::Queue TQueue>
  inline PointsHost<NDim> read_output(TQueue&, const std::string& file_path) {
    return read_output(Dim<NDim>{}, file_path);
  }

}  // namespace clue
