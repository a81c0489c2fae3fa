// Written against upstream openntc's public C++ API (README.md:54-112): it must compile
// unchanged against include/libopenntc/ and run on libontc.so.
//   usage: upstream_api_example <manifest.json> <out.ntc> <steps>
#include <libopenntc/libopenntc.h>
#include <libopenntc/openntc_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>

using namespace openntc;

int main(int argc, char** argv)
{
  if (argc < 4) return 2;
  Context ctx;
  ContextInitInfo init = {.profile_ = Profile::Bpp_0_5};
  if (ctx.Init(init) != Result::Success) return 3;
  if (ctx.LoadManifest(argv[1]) != Result::Success) return 4;
  TrainInfo train = {.quality_ = Quality::Low, .grids_per_batch_ = 1};
  ctx.BeginTraining(train);
  // upstream's GUI trains in chunks of 128 (openntc-gui/main.cpp:313); shorten the run
  ontc_train_options o = {};
  o.steps_override = std::atoi(argv[3]);
  ontc_set_train_options(ctx.Handle(), &o);
  TrainProgress p{};
  do {
    p = ctx.Train(128);
  } while (p.phase_ == TrainPhase::TrainInProgress);
  if (p.phase_ != TrainPhase::TrainComplete) return 5;

  EvalResults eval = ctx.Eval();
  std::cout << "PSNR: " << eval.psnr_ << " dB" << std::endl;
  if (Dump(argv[2], ctx.GetCompressedData()) != Result::Success) return 6;

  FileData file;
  if (Load(argv[2], file) != Result::Success) return 7;
  const CompressedData& cd = file.Data();
  NTCConstants consts;
  FillNTCConstants(cd, consts);
  std::cout << "levels " << cd.level_count_ << " dim " << consts.dim_ << " channels " << consts.channel_count_
            << " decoder " << cd.decoder_size_ << " bytes" << std::endl;
  if (ctx.decoder_host_ == nullptr || ctx.decoder_size_ != cd.decoder_size_) return 8;
  return 0;
}
