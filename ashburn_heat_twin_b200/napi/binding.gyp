{
  "targets": [
    {
      "target_name": "ahx_napi",
      "sources": ["ahx_napi.cc"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/..", "-lahx", "-Wl,-rpath,<(module_root_dir)/.."],
      "cflags_cc": ["-std=c++17", "-O2"],
      "defines": ["NAPI_VERSION=8"]
    }
  ]
}
