// A reference-style driver compiled against include/svg_b200.hpp: the steps
// of the reference's SAVING_SVG and TEST_SVG / TEST_SVG_MSAD mains
// (kernel.cu:17-105, 288-402, 404-455) with the interactive prompts replaced
// by a query file, so a test can run it and compare its output.
//
//   svg_driver in.obj K queries.txt
// writes in.svg next to in.obj and prints, per query line,
//   "s t"                  -> sssd <s> <t> <dist> path <t> ... <s>
//   "m n v0 w0 ... vn wn"  -> msad <n> then one line per vertex: <v> <dist> <srcId> <parent>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "svg_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 4) {
        std::cerr << "usage: svg_driver in.obj K queries.txt" << std::endl;
        return 2;
    }
    try {
        Mesh mesh, d_mesh;
        if (!mesh.LoadFromFile(argv[1])) {
            std::cerr << "cannot open " << argv[1] << std::endl;
            return 1;
        }
        mesh.copyToGPU(&d_mesh);

        SVG svg;
        svg.AssignMesh(&mesh, &d_mesh);
        svg.SetParameters(std::stoi(argv[2]), 10, 2);
        svg.Allocation();
        svg.ConstructSVG();
        svg.Free();
        svg.CopySVGToHost();

        std::string svgFileName = argv[1];
        svgFileName = svgFileName.substr(0, svgFileName.rfind('.')) + ".svg";
        svg.SaveSVGToFile(svgFileName.c_str());
        long long edges = 0;
        for (int v = 0; v < mesh.vertNum; ++v) edges += svg.Degree(v);
        std::printf("built %d vertices %lld edges\n", mesh.vertNum, edges);

        std::vector<SVG::GraphDistInfo> infos((size_t)mesh.vertNum);
        PriorityQueuesWithHandle<int> pq(mesh.vertNum);
        std::vector<PriorityQueuesWithHandle<int>::PQItem> pqBuf((size_t)mesh.vertNum + 1);
        pq.AssignMemory(pqBuf.data(), mesh.vertNum);

        std::ifstream qf(argv[3]);
        std::string line;
        while (std::getline(qf, line)) {
            std::istringstream in(line);
            std::string kind;
            in >> kind;
            if (kind == "m") {
                int n = 0;
                in >> n;
                std::vector<int> src((size_t)n);
                std::vector<double> w((size_t)n);
                for (int i = 0; i < n; ++i) in >> src[(size_t)i] >> w[(size_t)i];
                svg.SolveMSAD(src.data(), w.data(), n, mesh, infos.data(), pq);
                std::printf("msad %d\n", n);
                for (int v = 0; v < mesh.vertNum; ++v)
                    std::printf("%d %.17g %d %d\n", v, infos[(size_t)v].dist, infos[(size_t)v].srcId,
                                infos[(size_t)v].pathParentIndex);
            } else if (!kind.empty()) {
                int s = std::stoi(kind), t = -1;
                in >> t;
                svg.SolveSSSD(s, t, mesh, infos.data(), pq);
                std::printf("sssd %d %d %.17g path", s, t, infos[(size_t)t].dist);
                if (infos[(size_t)t].dist < DBL_MAX) {
                    int v = t;
                    while (v != s) {
                        std::printf(" %d", v);
                        v = infos[(size_t)v].pathParentIndex;
                    }
                    std::printf(" %d", s);
                }
                std::printf("\n");
                for (auto& gi : infos) gi = SVG::GraphDistInfo();  // kernel.cu:83-91
                pq.clear();
            }
        }
        svg.FreeSVGStructure();
        mesh.clear();
        d_mesh.clearGPU();
    } catch (const svg_b200::Error& e) {
        std::cerr << "svg_b200 error " << (int)e.code << ": " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
