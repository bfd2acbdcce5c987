// Test infrastructure: bounded-sample timing of the ExaCA reference's CPU path (OpenMP dispatch via
// the project's shims) for the CPU baseline. It performs the reference's own initialisation and step
// calls in RunProgram_Reduced's order (src/runCA.cpp:38-342, one rank, one layer, problem type C)
// and times Nucleation + CellCapture (+ IntermediateOutputAndCheck every 1000 cycles) over
// consecutive samples of `cycles_per_sample` cycles each with a steady clock. It prints one JSON
// object with the time of every sample.
//
//   ref_bench <input file> <samples> <cycles_per_sample> [dump file]
//
// With a dump file, the final GrainID and CellType (int32, LocalDomainSize each, in that order)
// are written there raw. Built with Serial dispatch (ref_bench_serial) this pins the restatement
// at a given cycle on domains too large for a complete reference run.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "CAfunctions.hpp"
#include "CAinitialize.hpp"
#include "CAtypes.hpp"
#include "CAupdate.hpp"

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: ref_bench <input file> <samples> <cycles_per_sample> [dump file]\n");
        return 2;
    }
    std::string input = argv[1];
    int samples = std::atoi(argv[2]);
    int per_sample = std::atoi(argv[3]);
    int id = 0, np = 1;
    int argc0 = 1;
    Kokkos::initialize(argc0, argv);
    {
        auto t_init0 = std::chrono::steady_clock::now();
        int nx, ny, nz, DecompositionStrategy, NumberOfLayers, LayerHeight, TempFilesInSeries;
        int NSpotsX, NSpotsY, SpotOffset, SpotRadius;
        unsigned int NumberOfTemperatureDataPoints = 0;
        bool ExtraWalls = false;
        int PrintDebug;
        bool PrintMisorientation, PrintFullOutput, RemeltingYN, UseSubstrateFile;
        float SubstrateGrainSpacing;
        double HT_deltax, deltax, deltat, FractSurfaceSitesActive, G, R, AConst, BConst, CConst, DConst,
            FreezingRange, NMax, dTN, dTsigma;
        std::string SubstrateFileName, temppath, tempfile, SimulationType, OutputFile, GrainOrientationFile,
            PathToOutput;
        std::vector<std::string> temp_paths;
        InputReadFromFile(id, input, SimulationType, DecompositionStrategy, AConst, BConst, CConst, DConst,
                          FreezingRange, deltax, NMax, dTN, dTsigma, OutputFile, GrainOrientationFile, temppath,
                          tempfile, TempFilesInSeries, temp_paths, ExtraWalls, HT_deltax, RemeltingYN, deltat,
                          NumberOfLayers, LayerHeight, SubstrateFileName, SubstrateGrainSpacing, UseSubstrateFile,
                          G, R, nx, ny, nz, FractSurfaceSitesActive, PathToOutput, PrintDebug, PrintMisorientation,
                          PrintFullOutput, NSpotsX, NSpotsY, SpotOffset, SpotRadius);
        if (SimulationType != "C") {
            std::fprintf(stderr, "ref_bench handles problem type C only\n");
            return 2;
        }
        int ProcessorsInXDirection, ProcessorsInYDirection, MyXSlices, MyXOffset, MyYSlices, MyYOffset;
        int NRN, NRS, NRE, NRW, NRNE, NRNW, NRSE, NRSW;
        ViewI_H NeighborX_H(Kokkos::ViewAllocateWithoutInitializing("NeighborX"), 26);
        ViewI_H NeighborY_H(Kokkos::ViewAllocateWithoutInitializing("NeighborY"), 26);
        ViewI_H NeighborZ_H(Kokkos::ViewAllocateWithoutInitializing("NeighborZ"), 26);
        ViewI2D_H ItList_H(Kokkos::ViewAllocateWithoutInitializing("ItList"), 9, 26);
        float XMin, YMin, ZMin, XMax, YMax, ZMax;
        std::vector<float> ZMinLayer(NumberOfLayers), ZMaxLayer(NumberOfLayers);
        std::vector<int> FinishTimeStep(NumberOfLayers), FirstValue(NumberOfLayers), LastValue(NumberOfLayers);
        std::vector<double> RawData(1);
        ParallelMeshInit(DecompositionStrategy, NeighborX_H, NeighborY_H, NeighborZ_H, ItList_H, SimulationType, id,
                         np, MyXSlices, MyYSlices, MyXOffset, MyYOffset, NRN, NRS, NRE, NRW, NRNE, NRNW, NRSE, NRSW,
                         deltax, HT_deltax, nx, ny, nz, ProcessorsInXDirection, ProcessorsInYDirection, temp_paths,
                         XMin, XMax, YMin, YMax, ZMin, ZMax, FreezingRange, LayerHeight, NumberOfLayers,
                         TempFilesInSeries, NumberOfTemperatureDataPoints, ZMinLayer.data(), ZMaxLayer.data(),
                         FirstValue.data(), LastValue.data(), RawData);
        long LocalDomainSize = (long)MyXSlices * MyYSlices * nz;
        ViewI_H CritTimeStep(Kokkos::ViewAllocateWithoutInitializing("CritTimeStep"), LocalDomainSize);
        ViewI_H LayerID(Kokkos::ViewAllocateWithoutInitializing("LayerID"), LocalDomainSize);
        ViewF_H UndercoolingChange(Kokkos::ViewAllocateWithoutInitializing("UndercoolingChange"), LocalDomainSize);
        ViewF_H UndercoolingCurrent(Kokkos::ViewAllocateWithoutInitializing("UndercoolingCurrent"), LocalDomainSize);
        std::vector<char> MeltedStore(LocalDomainSize);
        bool *Melted = reinterpret_cast<bool *>(MeltedStore.data());
        int ZBound_Low = -1, ZBound_High = -1, nzActive = -1;
        TempInit_DirSolidification(G, R, id, MyXSlices, MyYSlices, MyXOffset, MyYOffset, deltax, deltat, nx, ny, nz,
                                   CritTimeStep, UndercoolingChange, UndercoolingCurrent, Melted, nzActive,
                                   ZBound_Low, ZBound_High, LayerID);
        long LocalActiveDomainSize = (long)MyXSlices * MyYSlices * nzActive;
        int NGrainOrientations = 10000;
        ViewF_H GrainUnitVector(Kokkos::ViewAllocateWithoutInitializing("GrainUnitVector"), 9 * NGrainOrientations);
        ViewI_H GrainOrientation(Kokkos::ViewAllocateWithoutInitializing("GrainOrientation"), NGrainOrientations);
        OrientationInit(id, NGrainOrientations, GrainOrientation, GrainUnitVector, GrainOrientationFile);
        ViewI_H GrainID(Kokkos::ViewAllocateWithoutInitializing("GrainID"), LocalDomainSize);
        ViewI_H CellType(Kokkos::ViewAllocateWithoutInitializing("CellType"), LocalDomainSize);
        ViewF_H DiagonalLength(Kokkos::ViewAllocateWithoutInitializing("DiagonalLength"), LocalActiveDomainSize);
        // 64-bit size: 26 * cells exceeds int32 for the largest domains
        ViewF_H CritDiagonalLength(Kokkos::ViewAllocateWithoutInitializing("CritDiagonalLength"),
                                   26L * LocalActiveDomainSize);
        ViewF_H DOCenter(Kokkos::ViewAllocateWithoutInitializing("DOCenter"), 3L * LocalActiveDomainSize);
        int PossibleNuclei, NextLayer_FirstNucleatedGrainID;
        SubstrateInit_ConstrainedGrowth(FractSurfaceSitesActive, MyXSlices, MyYSlices, nx, ny, nz, MyXOffset,
                                        MyYOffset, id, np, CellType, GrainID);
        GrainInit(-1, NGrainOrientations, DecompositionStrategy, nz, (int)LocalActiveDomainSize, MyXSlices, MyYSlices,
                  MyXOffset, MyYOffset, id, np, NRN, NRS, NRE, NRW, NRNE, NRNW, NRSE, NRSW, ItList_H, NeighborX_H,
                  NeighborY_H, NeighborZ_H, GrainOrientation, GrainUnitVector, DiagonalLength, CellType, GrainID,
                  CritDiagonalLength, DOCenter, CritTimeStep, deltax, NMax, NextLayer_FirstNucleatedGrainID,
                  PossibleNuclei, ZBound_High, ZBound_Low);
        ViewI_H NucleationTimes(Kokkos::ViewAllocateWithoutInitializing("NucleationTimes"), PossibleNuclei);
        ViewI_H NucleiLocation(Kokkos::ViewAllocateWithoutInitializing("NucleiLocation"), PossibleNuclei);
        NucleiInit(DecompositionStrategy, MyXSlices, MyYSlices, nz, id, dTN, dTsigma, NRN, NRS, NRE, NRW, NRNE, NRNW,
                   NRSE, NRSW, NucleiLocation, NucleationTimes, CellType, GrainID, CritTimeStep, UndercoolingChange);
        AConst = AConst * deltat / deltax;
        BConst = BConst * deltat / deltax;
        CConst = CConst * deltat / deltax;
        int BufSizeX = MyXSlices, BufSizeY = 0, BufSizeZ = nzActive;
        Buffer2D BS(Kokkos::ViewAllocateWithoutInitializing("BufferSouthSend"), BufSizeX * BufSizeZ, 5);
        Buffer2D BN(Kokkos::ViewAllocateWithoutInitializing("BufferNorthSend"), BufSizeX * BufSizeZ, 5);
        Buffer2D BE, BW, BNE, BNW, BSE, BSW;
        ViewI SteeringVector(Kokkos::ViewAllocateWithoutInitializing("SteeringVector"), LocalActiveDomainSize);
        ViewI_H numSteer_H(Kokkos::ViewAllocateWithoutInitializing("SteeringVectorSize"), 1);
        numSteer_H(0) = 0;
        ViewI numSteer_G = numSteer_H;
        double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_init0).count();

        int cycle = 0, nn = 0, XSwitch = 0;
        int layernumber = 0;
        std::string st = SimulationType;
        std::vector<double> sample_s;
        for (int smp = 0; smp < samples && XSwitch == 0; smp++) {
            auto t0 = std::chrono::steady_clock::now();
            for (int q = 0; q < per_sample && XSwitch == 0; q++) {
                cycle++;
                Nucleation(MyXSlices, MyYSlices, MyXOffset, MyYOffset, cycle, nn, CellType, NucleiLocation,
                           NucleationTimes, GrainID, GrainOrientation, DOCenter, NeighborX_H, NeighborY_H,
                           NeighborZ_H, GrainUnitVector, CritDiagonalLength, DiagonalLength, NGrainOrientations,
                           PossibleNuclei, ZBound_Low, layernumber, LayerID);
                CellCapture(np, cycle, DecompositionStrategy, (int)LocalActiveDomainSize, (int)LocalDomainSize,
                            MyXSlices, MyYSlices, AConst, BConst, CConst, DConst, MyXOffset, MyYOffset, ItList_H,
                            NeighborX_H, NeighborY_H, NeighborZ_H, CritTimeStep, UndercoolingCurrent,
                            UndercoolingChange, GrainUnitVector, CritDiagonalLength, DiagonalLength,
                            GrainOrientation, CellType, DOCenter, GrainID, NGrainOrientations, BW, BE, BN, BS, BNE,
                            BNW, BSE, BSW, BufSizeX, BufSizeY, ZBound_Low, nzActive, nz, layernumber, LayerID,
                            SteeringVector, numSteer_G, numSteer_H);
                if (cycle % 1000 == 0)
                    IntermediateOutputAndCheck(id, cycle, MyXSlices, MyYSlices, (int)LocalDomainSize,
                                               (int)LocalActiveDomainSize, nn, XSwitch, CellType, CritTimeStep, st,
                                               FinishTimeStep.data(), layernumber, NumberOfLayers, ZBound_Low,
                                               LayerID);
            }
            sample_s.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        }
        if (argc > 4) {
            FILE *f = std::fopen(argv[4], "wb");
            if (!f || std::fwrite(GrainID.data(), sizeof(int), LocalDomainSize, f) != (size_t)LocalDomainSize ||
                std::fwrite(CellType.data(), sizeof(int), LocalDomainSize, f) != (size_t)LocalDomainSize) {
                std::fprintf(stderr, "cannot write %s\n", argv[4]);
                return 1;
            }
            std::fclose(f);
        }
        int threads = 1;
#ifdef EXACA_SHIM_OPENMP
        threads = omp_get_max_threads();
#endif
        std::printf("{\"cycles\": %d, \"cycles_per_sample\": %d, \"active_domain_cells\": %ld, \"init_s\": %.3f, "
                    "\"threads\": %d, \"sample_s\": [",
                    cycle, per_sample, LocalActiveDomainSize, init_s, threads);
        for (size_t q = 0; q < sample_s.size(); q++)
            std::printf("%s%.6f", q ? ", " : "", sample_s[q]);
        std::printf("]}\n");
    }
    Kokkos::finalize();
    return 0;
}
