{
  "targets": [
    {
      "target_name": "tpo_napi",
      "sources": ["tpo_napi.cc"],
      "include_dirs": ["../../include", "."],
      "cflags_cc": ["-std=c++17", "-O2"],
      "libraries": ["-L<(module_root_dir)/..", "-ltpo", "-Wl,-rpath,<(module_root_dir)/.."]
    }
  ]
}
